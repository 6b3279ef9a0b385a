// bp_engine.cpp -- context, device memory, solver drivers and the C ABI.
//
// One context = one device + one stream + a growing device arena that is
// reused across calls (time steps), so repeated solves do not reallocate.
// The drivers only enqueue work; all scalar decisions (alpha, beta,
// convergence, Picard stop) are taken on the device.  The host reads two
// counters per PCG check chunk and one per Picard iteration, one chunk
// behind the device, to know when to stop enqueuing.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "bp_b200.h"
#include "bp_common.h"
#include "bp_kernels.h"
#include "bp_plan.h"

struct bp_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  std::map<std::string, std::pair<void*, size_t>> arena;
  bp::Counters* h_cnt = nullptr;   // pinned, [2] slots
  cudaEvent_t ev[2] = {nullptr, nullptr};
  cudaEvent_t t0 = nullptr, t1 = nullptr, t2 = nullptr, t3 = nullptr;
  int num_sms = 0;
  int grid_cap = 0;
  bool tables_ready = false;
};

namespace {

using namespace bp;

struct CudaError {
  cudaError_t e;
  const char* what;
};

#define CK(call)                                           \
  do {                                                     \
    cudaError_t e_ = (call);                               \
    if (e_ != cudaSuccess) throw CudaError{e_, #call};     \
  } while (0)

template <typename T>
T* arena_get(bp_ctx* c, const char* name, size_t count) {
  size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
  bytes = (bytes + 255) / 256 * 256;
  auto it = c->arena.find(name);
  if (it != c->arena.end() && it->second.second >= bytes) return static_cast<T*>(it->second.first);
  if (it != c->arena.end()) {
    CK(cudaStreamSynchronize(c->stream));
    CK(cudaFree(it->second.first));
    c->arena.erase(it);
  }
  void* p = nullptr;
  CK(cudaMalloc(&p, bytes));
  c->arena[name] = {p, bytes};
  return static_cast<T*>(p);
}

template <typename T>
void upload(bp_ctx* c, T* dst, const std::vector<T>& src) {
  if (!src.empty())
    CK(cudaMemcpyAsync(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, c->stream));
}

// Device arrays of a plan.  `with_cells` = element data needed.
DevView make_view(bp_ctx* c, const HostPlan& p, bool with_cells, bool mixed) {
  DevView v;
  std::memset(&v, 0, sizeof(v));
  v.nz = p.nz; v.ncols = p.ncols; v.nnodes = p.nnodes; v.npad = p.npad;
  v.ncells = p.ncells; v.nelem = p.nelem; v.ninst = p.ninst; v.ntiles = p.ntiles;
  int anyd = 0;
  for (uint8_t m : p.dmask) anyd |= (m != 0);
  v.any_dirichlet = anyd;
  const size_t np = (size_t)p.npad;
  InstParams* inst = arena_get<InstParams>(c, "inst", p.ninst);
  upload(c, inst, p.inst);
  v.inst = inst;
  v.st = arena_get<InstState>(c, "st", p.ninst);
  v.cnt = arena_get<Counters>(c, "cnt", 1);
  int* col_inst = arena_get<int>(c, "col_inst", p.ncols); upload(c, col_inst, p.col_inst); v.col_inst = col_inst;
  int* col_nbr = arena_get<int>(c, "col_nbr", p.col_nbr.size()); upload(c, col_nbr, p.col_nbr); v.col_nbr = col_nbr;
  int* col_cells = arena_get<int>(c, "col_cells", p.col_cells.size()); upload(c, col_cells, p.col_cells); v.col_cells = col_cells;
  int* col_ij = arena_get<int>(c, "col_ij", p.col_ij.size()); upload(c, col_ij, p.col_ij); v.col_ij = col_ij;
  double* col_beta = arena_get<double>(c, "col_beta", p.col_beta.size()); upload(c, col_beta, p.col_beta); v.col_beta = col_beta;
  double2* load = arena_get<double2>(c, "load", p.load.size()); upload(c, load, p.load); v.load = load;
  uint8_t* dmask = arena_get<uint8_t>(c, "dmask", p.dmask.size()); upload(c, dmask, p.dmask); v.dmask = dmask;
  if (with_cells) {
    int* a = arena_get<int>(c, "cell_inst", p.cell_inst.size()); upload(c, a, p.cell_inst); v.cell_inst = a;
    a = arena_get<int>(c, "cell_ij", p.cell_ij.size()); upload(c, a, p.cell_ij); v.cell_ij = a;
    a = arena_get<int>(c, "cell_cols", p.cell_cols.size()); upload(c, a, p.cell_cols); v.cell_cols = a;
    double* d = arena_get<double>(c, "cell_s", p.cell_s.size()); upload(c, d, p.cell_s); v.cell_s = d;
    d = arena_get<double>(c, "cell_h", p.cell_h.size()); upload(c, d, p.cell_h); v.cell_h = d;
    d = arena_get<double>(c, "cell_beta", p.cell_beta.size()); upload(c, d, p.cell_beta); v.cell_beta = d;
    d = arena_get<double>(c, "flwafact", p.flwafact.size()); upload(c, d, p.flwafact); v.flwafact = d;
    v.qp = arena_get<double>(c, "qp", (size_t)p.nelem * 80);
    v.efvs = arena_get<double>(c, "efvs", p.nelem);
    v.badj = arena_get<double>(c, "badj", 4 * np);
  }
  int* ts = arena_get<int>(c, "tile_start", p.tile_start.size()); upload(c, ts, p.tile_start); v.tile_start = ts;
  int* ti = arena_get<int>(c, "tile_inst", p.tile_inst.size()); upload(c, ti, p.tile_inst); v.tile_inst = ti;
  v.A = arena_get<double2>(c, "A", 2 * 27 * np);
  v.x = arena_get<double2>(c, "x", np);
  v.b = arena_get<double2>(c, "b", np);
  v.r = arena_get<double2>(c, "r", np);
  v.d0 = arena_get<double2>(c, "d0", np);
  v.d1 = arena_get<double2>(c, "d1", np);
  v.q = arena_get<double2>(c, "q", np);
  v.Az = arena_get<double2>(c, "Az", np);
  v.Dinv = arena_get<double2>(c, "Dinv", np);
  v.usav = arena_get<double2>(c, "usav", np);
  if (mixed) {
    v.A32 = arena_get<float2>(c, "A32", 2 * 27 * np);
    v.scale = arena_get<double2>(c, "scale", np);
    v.y32 = arena_get<float2>(c, "y32", np);
    v.r32 = arena_get<float2>(c, "r32", np);
    v.p32a = arena_get<float2>(c, "p32a", np);
    v.p32b = arena_get<float2>(c, "p32b", np);
    v.q32 = arena_get<float2>(c, "q32", np);
  }
  v.partials = arena_get<double>(c, "partials", 2 * (size_t)std::max(p.ntiles, 1));
  v.tile_counter = arena_get<unsigned>(c, "tile_counter", p.ninst);
  CK(cudaMemsetAsync(v.tile_counter, 0, sizeof(unsigned) * p.ninst, c->stream));
  return v;
}

void init_state(bp_ctx* c, const DevView& v, const HostPlan& p, bool picard, bool pcg) {
  const int ninst = p.ninst;
  std::vector<InstState> st(ninst);
  int live = 0;
  for (int b = 0; b < ninst; ++b) {
    InstState& s = st[b];
    std::memset(&s, 0, sizeof(s));
    const bool empty = p.inst[b].node_end == p.inst[b].node_begin;
    // no active vertex at all: count_nonzeros_3d = 0, velocity zero
    // (glissade_velo_higher.F90:3191-3220)
    s.status = empty ? BP_ZERO_MATRIX : BP_OK;
    s.picard_active = (picard && !empty) ? 1 : 0;
    s.pcg_active = (pcg && !empty) ? 1 : 0;
    s.refine_active = s.pcg_active;
    s.pcg_iter = 1;
    s.rz = 1.0;
    s.rz_old = 1.0;
    s.err = -1.0;
    live += empty ? 0 : 1;
  }
  CK(cudaMemcpyAsync(v.st, st.data(), sizeof(InstState) * ninst, cudaMemcpyHostToDevice, c->stream));
  Counters h{};
  h.picard_active = picard ? live : 0;
  h.pcg_active = pcg ? live : 0;
  h.refine_active = pcg ? live : 0;
  CK(cudaMemcpyAsync(v.cnt, &h, sizeof(h), cudaMemcpyHostToDevice, c->stream));
}

// Copy the counters to pinned slot `slot` and record its event.
void snapshot(bp_ctx* c, const DevView& v, int slot) {
  CK(cudaMemcpyAsync(&c->h_cnt[slot], v.cnt, sizeof(Counters), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaEventRecord(c->ev[slot], c->stream));
}

Counters wait_snapshot(bp_ctx* c, int slot) {
  CK(cudaEventSynchronize(c->ev[slot]));
  return c->h_cnt[slot];
}

int max_pcg_iters(const HostPlan& p) {
  int m = 1;
  for (const auto& ip : p.inst) m = std::max(m, ip.pcg_maxiters);
  return m;
}

// FP64 PCG (standard or Chronopoulos-Gear) for all instances with
// pcg_active, starting after MV_INIT.  Iterations run in chunks that end
// at a convergence check; the host polls one chunk behind.
void run_pcg_fp64(bp_ctx* c, const DevView& v, const HostPlan& p) {
  const int variant = p.inst[0].variant;
  const int ncheck = std::max(1, p.inst[0].ncheck);
  const int maxit = max_pcg_iters(p);
  int n = 1;
  if (variant == 3) {
    launch_mv(MV_CG_FIRST, v, c->stream);
    launch_cg_first_update(v, c->stream);
    n = 2;
  }
  int chunk = 0;
  while (n <= maxit + 1) {
    // iterations n .. next multiple of ncheck
    do {
      const bool check = (n % ncheck) == 0;
      if (variant == 3) {
        launch_mv(MV_CG1, v, c->stream);
        launch_cg_update(check, v, c->stream);
      } else {
        launch_mv(MV_STD_A, v, c->stream);
        launch_std_update(check, v, c->stream);
      }
      if (check) launch_mv(MV_CHECK, v, c->stream);
      ++n;
    } while ((n - 1) % ncheck != 0 && n <= maxit + 1);
    snapshot(c, v, chunk & 1);
    if (chunk >= 1) {
      const Counters h = wait_snapshot(c, (chunk - 1) & 1);
      if (h.pcg_active <= 0) break;
    }
    ++chunk;
  }
  CK(cudaGetLastError());
}

// Mixed precision linear solve: FP64 refinement around FP32 inner CG.
void run_mixed(bp_ctx* c, const DevView& v, const HostPlan& p) {
  launch_mixed_setup(v, c->stream);
  const int maxit = max_pcg_iters(p);
  for (int ref = 0; ref < 24; ++ref) {
    CK(cudaMemsetAsync(&v.cnt->pcg_active, 0, sizeof(int), c->stream));
    launch_refine_resid(v, c->stream);
    snapshot(c, v, 0);
    const Counters h = wait_snapshot(c, 0);
    if (h.refine_active <= 0) break;
    int chunk = 0, it = 0;
    const int inner_chunk = 8;
    while (it < maxit) {
      for (int j = 0; j < inner_chunk; ++j) launch_inner(v, c->stream);
      it += inner_chunk;
      snapshot(c, v, chunk & 1);
      if (chunk >= 1) {
        const Counters hh = wait_snapshot(c, (chunk - 1) & 1);
        if (hh.pcg_active <= 0) break;
      }
      ++chunk;
    }
    launch_refine_update(v, c->stream);
  }
  CK(cudaGetLastError());
}

// Linear solve of the currently assembled system for active instances.
void linear_solve(bp_ctx* c, const DevView& v, const HostPlan& p) {
  if (p.inst[0].precision == BP_MIXED) {
    run_mixed(c, v, p);
  } else {
    launch_mv(MV_INIT, v, c->stream);
    run_pcg_fp64(c, v, p);
  }
}

int fill_stats(const InstState& s, bp_stats* st) {
  if (!st) return s.status;
  std::memset(st, 0, sizeof(*st));
  st->status = s.status;
  st->picard_iters = s.picard_iter;
  st->pcg_iters_total = s.pcg_iters_total;
  st->pcg_iters_last = s.pcg_iters_last;
  st->refine_steps_total = s.refine_steps_total;
  st->converged = s.picard_converged;
  st->pcg_err_last = s.err;
  st->resid_velo = s.resid_velo;
  st->L2_norm = s.L2_norm;
  st->L2_norm_relative = s.L2_rel;
  return s.status;
}

int final_status(const InstState& s) {
  if (s.status != BP_OK) return s.status;
  if (!s.picard_converged) return BP_WARN_PICARD_NOT_CONVERGED;
  if (!s.pcg_converged) return BP_WARN_PCG_NOT_CONVERGED;
  return BP_OK;
}

int solve_batch(bp_ctx* c, int n, const bp_inputs* in, double* const* uvel,
                double* const* vvel, double* const* efvs, bp_stats* stats) {
  HostPlan p;
  std::string err;
  if (!build_plan(in, n, &p, &err)) {
    c->err = err;
    return BP_ERR_ARGS;
  }
  const bool mixed = p.inst[0].precision == BP_MIXED;
  CK(cudaEventRecord(c->t0, c->stream));
  DevView v = make_view(c, p, true, mixed);
  std::vector<double2> x(p.npad, double2{0.0, 0.0});
  for (int b = 0; b < n; ++b) gather_velocity(p, b, uvel[b], vvel[b], x.data());
  CK(cudaMemcpyAsync(v.x, x.data(), sizeof(double2) * p.npad, cudaMemcpyHostToDevice, c->stream));
  init_state(c, v, p, true, false);
  CK(cudaEventRecord(c->t1, c->stream));
  int max_picard = 1;
  for (const auto& ip : p.inst) max_picard = std::max(max_picard, ip.maxiter_nonlinear);
  for (int it = 0; it < max_picard; ++it) {
    launch_picard_begin(v, c->stream);
    launch_save_usav(v, c->stream);
    launch_assemble(v, c->stream);
    linear_solve(c, v, p);
    launch_picard_check(v, c->stream);
    snapshot(c, v, 0);
    const Counters h = wait_snapshot(c, 0);
    if (h.picard_active <= 0) break;
  }
  CK(cudaEventRecord(c->t2, c->stream));
  CK(cudaMemcpyAsync(x.data(), v.x, sizeof(double2) * p.npad, cudaMemcpyDeviceToHost, c->stream));
  std::vector<double> ef;
  if (efvs) {
    ef.resize(std::max(p.nelem, 1));
    if (p.nelem > 0)
      CK(cudaMemcpyAsync(ef.data(), v.efvs, sizeof(double) * p.nelem, cudaMemcpyDeviceToHost, c->stream));
  }
  std::vector<InstState> st(n);
  CK(cudaMemcpyAsync(st.data(), v.st, sizeof(InstState) * n, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaEventRecord(c->t3, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaGetLastError());
  float ms_up = 0, ms_solve = 0, ms_tot = 0;
  cudaEventElapsedTime(&ms_up, c->t0, c->t1);
  cudaEventElapsedTime(&ms_solve, c->t1, c->t2);
  cudaEventElapsedTime(&ms_tot, c->t0, c->t3);
  int worst = BP_OK;
  for (int b = 0; b < n; ++b) {
    scatter_velocity(p, b, x.data(), uvel[b], vvel[b]);
    if (efvs && efvs[b]) scatter_efvs(p, b, ef.data(), efvs[b]);
    if (stats) {
      fill_stats(st[b], &stats[b]);
      stats[b].status = final_status(st[b]);
      stats[b].ms_upload = ms_up;
      stats[b].ms_pcg = ms_solve;
      stats[b].ms_total = ms_tot;
    }
    const int s = final_status(st[b]);
    if (s != BP_OK && (worst == BP_OK || (s != BP_WARN_PCG_NOT_CONVERGED && s != BP_WARN_PICARD_NOT_CONVERGED)))
      worst = s;
  }
  return worst;
}

}  // namespace

// ----------------------------------------------------------------------
// C ABI
// ----------------------------------------------------------------------
extern "C" {

int bp_abi_version(void) { return BP_ABI_VERSION; }

int bp_create(int device, bp_ctx** out) {
  if (!out) return BP_ERR_ARGS;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return BP_ERR_NO_DEVICE;
  if (device < 0 || device >= ndev) return BP_ERR_ARGS;
  bp_ctx* c = new bp_ctx();
  c->device = device;
  try {
    CK(cudaSetDevice(device));
    CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    CK(cudaMallocHost((void**)&c->h_cnt, 2 * sizeof(bp::Counters)));
    for (auto& e : c->ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    CK(cudaEventCreate(&c->t0));
    CK(cudaEventCreate(&c->t1));
    CK(cudaEventCreate(&c->t2));
    CK(cudaEventCreate(&c->t3));
    CK(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device));
    CK(bp::upload_ref_tables());
    c->tables_ready = true;
  } catch (const CudaError& e) {
    std::fprintf(stderr, "bp_create: %s failed: %s\n", e.what, cudaGetErrorString(e.e));
    bp_destroy(c);
    return BP_ERR_CUDA;
  }
  *out = c;
  return BP_OK;
}

int bp_destroy(bp_ctx* c) {
  if (!c) return BP_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (auto& kv : c->arena) cudaFree(kv.second.first);
  if (c->h_cnt) cudaFreeHost(c->h_cnt);
  for (auto& e : c->ev)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : {c->t0, c->t1, c->t2, c->t3})
    if (e) cudaEventDestroy(e);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return BP_OK;
}

const char* bp_last_error(const bp_ctx* c) { return c ? c->err.c_str() : "no context"; }

#define GUARD_BEGIN                 \
  if (!c) return BP_ERR_ARGS;       \
  c->err.clear();                   \
  try {                             \
    CK(cudaSetDevice(c->device));
#define GUARD_END                                                     \
  }                                                                   \
  catch (const CudaError& e) {                                        \
    c->err = std::string(e.what) + ": " + cudaGetErrorString(e.e);    \
    return BP_ERR_CUDA;                                               \
  }

int bp_batch_solve(bp_ctx* c, int n, const bp_inputs* in, double* const* uvel,
                   double* const* vvel, double* const* efvs, bp_stats* stats) {
  GUARD_BEGIN
  if (n < 1 || !in || !uvel || !vvel) return BP_ERR_ARGS;
  return solve_batch(c, n, in, uvel, vvel, efvs, stats);
  GUARD_END
}

int bp_solve(bp_ctx* c, const bp_inputs* in, double* uvel, double* vvel,
             double* efvs, bp_stats* stats) {
  double* u[1] = {uvel};
  double* w[1] = {vvel};
  double* e[1] = {efvs};
  return bp_batch_solve(c, 1, in, u, w, efvs ? e : nullptr, stats);
}

int bp_pcg(bp_ctx* c, int nx, int ny, int nz, int periodic,
           const int* active_vertex, const double* Auu, const double* Auv,
           const double* Avu, const double* Avv, const double* bu,
           const double* bv, double* xu, double* xv, int precond, int variant,
           double tol, int maxiters, int ncheck, int precision, double* err,
           int* niters) {
  GUARD_BEGIN
  if (!active_vertex || !Auu || !Auv || !Avu || !Avv || !bu || !bv || !xu || !xv)
    return BP_ERR_ARGS;
  if (precond != 0 && precond != 1) {
    c->err = "bp_pcg: precond must be 0 or 1";
    return BP_ERR_ARGS;
  }
  HostPlan p;
  std::string e;
  if (!build_column_plan(nx, ny, nz, periodic, active_vertex, &p, &e)) {
    c->err = e;
    return BP_ERR_ARGS;
  }
  InstParams& ip = p.inst[0];
  ip.precond = precond;
  ip.variant = variant == 3 ? 3 : 2;
  ip.pcg_tol = tol;
  ip.pcg_maxiters = maxiters;
  ip.ncheck = ncheck > 0 ? ncheck : 5;
  ip.precision = precision;
  ip.inner_tol = 1.0e-4;
  const bool mixed = precision == BP_MIXED;
  DevView v = make_view(c, p, false, mixed);
  std::vector<double2> A(2 * 27 * (size_t)p.npad);
  gather_matrix(p, Auu, Auv, Avu, Avv, A.data());
  CK(cudaMemcpyAsync(v.A, A.data(), sizeof(double2) * A.size(), cudaMemcpyHostToDevice, c->stream));
  std::vector<double2> x(p.npad, double2{0, 0}), b(p.npad, double2{0, 0});
  gather_velocity(p, 0, xu, xv, x.data());
  gather_velocity(p, 0, bu, bv, b.data());
  CK(cudaMemcpyAsync(v.x, x.data(), sizeof(double2) * p.npad, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(v.b, b.data(), sizeof(double2) * p.npad, cudaMemcpyHostToDevice, c->stream));
  init_state(c, v, p, false, true);
  launch_dinv(v, precond, c->stream);
  launch_bb(v, c->stream);
  linear_solve(c, v, p);
  CK(cudaMemcpyAsync(x.data(), v.x, sizeof(double2) * p.npad, cudaMemcpyDeviceToHost, c->stream));
  InstState st;
  CK(cudaMemcpyAsync(&st, v.st, sizeof(st), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaGetLastError());
  scatter_velocity(p, 0, x.data(), xu, xv);
  if (err) *err = st.err;
  if (niters) *niters = mixed ? st.pcg_iters_total : st.pcg_iters_last;
  if (st.status != BP_OK) return st.status;
  return st.pcg_converged ? BP_OK : BP_WARN_PCG_NOT_CONVERGED;
  GUARD_END
}

int bp_matvec(bp_ctx* c, int nx, int ny, int nz, int periodic,
              const int* active_vertex, const double* Auu, const double* Auv,
              const double* Avu, const double* Avv, const double* xu,
              const double* xv, double* yu, double* yv) {
  GUARD_BEGIN
  if (!active_vertex || !Auu || !Auv || !Avu || !Avv || !xu || !xv || !yu || !yv)
    return BP_ERR_ARGS;
  HostPlan p;
  std::string e;
  if (!build_column_plan(nx, ny, nz, periodic, active_vertex, &p, &e)) {
    c->err = e;
    return BP_ERR_ARGS;
  }
  DevView v = make_view(c, p, false, false);
  std::vector<double2> A(2 * 27 * (size_t)p.npad);
  gather_matrix(p, Auu, Auv, Avu, Avv, A.data());
  CK(cudaMemcpyAsync(v.A, A.data(), sizeof(double2) * A.size(), cudaMemcpyHostToDevice, c->stream));
  std::vector<double2> x(p.npad, double2{0, 0});
  gather_velocity(p, 0, xu, xv, x.data());
  CK(cudaMemcpyAsync(v.x, x.data(), sizeof(double2) * p.npad, cudaMemcpyHostToDevice, c->stream));
  launch_matvec_plain(v, v.x, v.r, c->stream);
  CK(cudaMemcpyAsync(x.data(), v.r, sizeof(double2) * p.npad, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaGetLastError());
  const size_t tot = (size_t)nz * (nx - 1) * (ny - 1);
  std::memset(yu, 0, sizeof(double) * tot);
  std::memset(yv, 0, sizeof(double) * tot);
  scatter_vector(p, 0, x.data(), yu, yv);
  return BP_OK;
  GUARD_END
}

int bp_assemble(bp_ctx* c, const bp_inputs* in, const double* uvel,
                const double* vvel, double* Auu, double* Auv, double* Avu,
                double* Avv, double* bu, double* bv, double* efvs) {
  GUARD_BEGIN
  if (!in || !uvel || !vvel) return BP_ERR_ARGS;
  HostPlan p;
  std::string e;
  if (!build_plan(in, 1, &p, &e)) {
    c->err = e;
    return BP_ERR_ARGS;
  }
  DevView v = make_view(c, p, true, false);
  std::vector<double2> x(p.npad, double2{0, 0});
  gather_velocity(p, 0, uvel, vvel, x.data());
  CK(cudaMemcpyAsync(v.x, x.data(), sizeof(double2) * p.npad, cudaMemcpyHostToDevice, c->stream));
  init_state(c, v, p, true, false);
  launch_picard_begin(v, c->stream);
  launch_assemble(v, c->stream);
  std::vector<double2> A(2 * 27 * (size_t)p.npad), b(p.npad);
  std::vector<double> ef(std::max(p.nelem, 1));
  CK(cudaMemcpyAsync(A.data(), v.A, sizeof(double2) * A.size(), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(b.data(), v.b, sizeof(double2) * p.npad, cudaMemcpyDeviceToHost, c->stream));
  if (p.nelem > 0)
    CK(cudaMemcpyAsync(ef.data(), v.efvs, sizeof(double) * p.nelem, cudaMemcpyDeviceToHost, c->stream));
  InstState st;
  CK(cudaMemcpyAsync(&st, v.st, sizeof(st), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaGetLastError());
  scatter_matrix(p, A.data(), Auu, Auv, Avu, Avv);
  const size_t tot = (size_t)in->nz * (in->nx - 1) * (in->ny - 1);
  if (bu) std::memset(bu, 0, sizeof(double) * tot);
  if (bv) std::memset(bv, 0, sizeof(double) * tot);
  scatter_vector(p, 0, b.data(), bu, bv);
  if (efvs) scatter_efvs(p, 0, ef.data(), efvs);
  return st.status == BP_ZERO_MATRIX ? BP_ZERO_MATRIX : st.status;
  GUARD_END
}

}  // extern "C"
