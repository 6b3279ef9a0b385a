// bp_engine.cpp -- context, resident problems, solver drivers and the C ABI.
//
// A context is one device and one stream.  A problem is a compiled solve (or
// batch) resident in device memory: its plan arrays, matrix, vectors and the
// CUDA graphs of its PCG check chunks, reused across runs.  The drivers only
// enqueue work; every scalar decision (alpha, beta, convergence, Picard
// stop) is taken on the device.  The host reads a 16-byte counter snapshot
// once per check chunk, one chunk behind the device, to stop enqueuing.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <tuple>
#include <string>
#include <vector>

#include "bp_b200.h"
#include "bp_common.h"
#include "bp_guess.h"
#include "bp_kernels.h"
#include "bp_plan.h"

namespace {

// A learned guess that cannot run (no network loaded, or its launch failed).
struct GuessError {
  const char* what;
};

struct CudaError {
  cudaError_t e;
  const char* what;
};

#define CK(call)                                           \
  do {                                                     \
    cudaError_t e_ = (call);                               \
    if (e_ != cudaSuccess) throw CudaError{e_, #call};     \
  } while (0)

// Named device allocations that only grow.
struct Arena {
  std::map<std::string, std::pair<void*, size_t>> m;
  template <typename T>
  T* get(cudaStream_t s, const char* name, size_t count) {
    size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    bytes = (bytes + 255) / 256 * 256;
    auto it = m.find(name);
    if (it != m.end() && it->second.second >= bytes) return static_cast<T*>(it->second.first);
    if (it != m.end()) {
      CK(cudaStreamSynchronize(s));
      CK(cudaFree(it->second.first));
      m.erase(it);
    }
    void* p = nullptr;
    CK(cudaMalloc(&p, bytes));
    m[name] = {p, bytes};
    return static_cast<T*>(p);
  }
  void release() {
    for (auto& kv : m) cudaFree(kv.second.first);
    m.clear();
  }
};

// Event pairs around kernel launches, by category.
struct Timing {
  bool on = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pool;
  std::vector<int> cat;
  double ms[BP_NUM_KERNEL_CATEGORIES] = {0};
  int n[BP_NUM_KERNEL_CATEGORIES] = {0};
  void reset() {
    cat.clear();
    for (int i = 0; i < BP_NUM_KERNEL_CATEGORIES; ++i) { ms[i] = 0.0; n[i] = 0; }
  }
  void destroy() {
    for (auto& pr : pool) { cudaEventDestroy(pr.first); cudaEventDestroy(pr.second); }
    pool.clear();
  }
};

}  // namespace

struct bp_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  Arena arena;                     // for the one-shot entry points
  bp::Counters* h_cnt = nullptr;   // pinned, 2 slots
  cudaEvent_t ev[2] = {nullptr, nullptr};
  cudaEvent_t t0 = nullptr, t1 = nullptr, t2 = nullptr, t3 = nullptr;
  cudaEvent_t r0 = nullptr, r1 = nullptr;  // bp_timer_start / stop
  int num_sms = 0;
  int l2_max_persist = 0, l2_max_window = 0;  // bytes (0 = no persisting L2)
  // autotuner results: (node bucket, nz, storage, precision, PCG variant)
  // -> (minb, grid) of the residual kernels, (minb_k, grid_k) of the Krylov matvecs
  std::map<std::tuple<int, int, int, int, int>, std::array<int, 4>> tuned;
  bp::GuessNet* net = nullptr;     // the learned guess's network (bp_guess_load)
  int net_launches = 0;            // kernels the network launched (bp_guess_launches)
};

struct bp_problem {
  bp_ctx* c = nullptr;
  Arena own;
  Arena* arena = nullptr;
  bp::HostPlan plan;
  bp::DevView v;
  bool mixed = false;
  double2* x0 = nullptr;
  // DIVA: the starting 3-D velocity, point viscosities and traction, copied
  // into the working arrays at the start of every run
  double2* x3_0 = nullptr;
  double* eq3_0 = nullptr;
  double2* bt0 = nullptr;
  cudaGraphExec_t chunk_graph = nullptr;
  cudaGraphExec_t inner_graph = nullptr;
  // the device-resident Picard loop (one graph with nested WHILE nodes) and
  // its pass counters (Picard, PCG chunks); loop_state: 0 not built yet, 1
  // built, -1 unavailable (the host-driven loop runs)
  cudaGraphExec_t loop_graph = nullptr;
  int* loop_iter = nullptr;
  int loop_state = 0;
  bool use_graphs = true;
  Timing timing;
  bool tuned = false;
  unsigned long long* mv_nodes_dev = nullptr;
  unsigned long long mv_nodes[2] = {0, 0};
  std::vector<bp::InstState> state;
  float ms_upload = 0, ms_solve = 0;
  double h2d_bytes = 0, d2h_bytes = 0;
};

namespace {

using namespace bp;

double g_h2d = 0.0;  // bytes uploaded by the current call (single-threaded per context)

template <typename T>
void upload(cudaStream_t s, T* dst, const std::vector<T>& src) {
  if (!src.empty()) {
    CK(cudaMemcpyAsync(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, s));
    g_h2d += (double)src.size() * sizeof(T);
  }
}

// Allocate and upload the device arrays of a plan.
DevView make_view(Arena& a, cudaStream_t s, const HostPlan& p, bool with_cells, bool mixed) {
  DevView v;
  std::memset(&v, 0, sizeof(v));
  v.nz = p.nz; v.ncols = p.ncols; v.nnodes = p.nnodes; v.npad = p.npad;
  v.W = p.W; v.lsh = p.lsh;
  v.tile_threads = std::min(kTile, (p.W * p.nz + 31) / 32 * 32);
  v.solve2d = p.solve2d ? 1 : 0;
  v.l1l2 = p.l1l2 ? 1 : 0;
  v.diva = p.diva ? 1 : 0;
  v.nl = p.nz_out - 1;
  v.ncells = p.ncells; v.nelem = p.nelem; v.ninst = p.ninst; v.ntiles = p.ntiles;
  int anyd = 0;
  for (uint8_t m : p.dmask) anyd |= (m != 0);
  v.any_dirichlet = anyd;
  // systems assembled on the device are exactly symmetric: store half
  // (BP_MATRIX_STORAGE=full keeps whole rows, for the kernel sweep)
  const char* st_env = std::getenv("BP_MATRIX_STORAGE");
  v.sym = (with_cells && !(st_env && std::string(st_env) == "full")) ? 1 : 0;
  const size_t np = (size_t)p.npad;
#define UP(T, name, vec, field)                           \
  {                                                       \
    T* d_ = a.get<T>(s, name, (vec).size());              \
    upload(s, d_, vec);                                   \
    v.field = d_;                                         \
  }
  UP(InstParams, "inst", p.inst, inst);
  v.st = a.get<InstState>(s, "st", p.ninst);
  v.cnt = a.get<Counters>(s, "cnt", 1);
  UP(int, "col_inst", p.col_inst, col_inst);
  UP(int, "col_nbr", p.col_nbr, col_nbr);
  UP(int, "col_node", p.col_node, col_node);
  UP(int, "col_nbn", p.col_nbn, col_nbn);
  UP(int, "col_cells", p.col_cells, col_cells);
  UP(int, "col_ij", p.col_ij, col_ij);
  UP(double, "col_beta", p.col_beta, col_beta);
  UP(double, "col_h", p.col_h, col_h);
  if (p.any_sliding) UP(double, "col_slide", p.col_slide, col_slide);
  UP(double2, "load", p.load, load);
  UP(uint8_t, "dmask", p.dmask, dmask);
  if (with_cells) {
    UP(int, "cell_inst", p.cell_inst, cell_inst);
    UP(int, "cell_ij", p.cell_ij, cell_ij);
    UP(int, "cell_cols", p.cell_cols, cell_cols);
    UP(double, "cell_s", p.cell_s, cell_s);
    UP(double, "cell_h", p.cell_h, cell_h);
    UP(double, "cell_beta", p.cell_beta, cell_beta);
    UP(double, "flwafact", p.flwafact, flwafact);
    v.qp = a.get<double>(s, "qp", (size_t)p.nelem * 80);
    v.efvs = a.get<double>(s, "efvs", p.nefvs);
    // element-centric 3-D assembly (k_asm_elem + gather): the element blocks
    // of one assembly, 2 KiB per element, when they take at most 32 GiB and
    // a quarter of the free device memory; otherwise (or BP_ASM_ELEM=0) each
    // row integrates its incident elements itself.  Both give the same
    // matrix bitwise.
    if (!p.solve2d && p.nelem > 0) {
      const char* e = std::getenv("BP_ASM_ELEM");
      const size_t bytes = (size_t)p.nelem * 256 * sizeof(double);
      size_t free_b = 0, total_b = 0;
      if (!(e && e[0] == '0') && bytes <= ((size_t)32 << 30) &&
          cudaMemGetInfo(&free_b, &total_b) == cudaSuccess && bytes <= free_b / 4)
        v.Ke = a.get<double>(s, "Ke", (size_t)p.nelem * 256);
    }
    if (p.l1l2) {
      UP(double, "cell_flwa", p.cell_flwa, cell_flwa);
      UP(double, "cell_thck", p.cell_thck, cell_thck);
      UP(double, "cell_ds", p.cell_ds, cell_ds);
      UP(double, "col_ds", p.col_ds, col_ds);

      v.lw = a.get<double>(s, "l1l2_work", 4 * (size_t)v.nl * std::max(p.ncells, 1));
      v.x3 = a.get<double2>(s, "x3", (size_t)std::max(p.ncols, 1) * (v.nl + 1));
    }
    if (p.diva) {
      UP(double, "cell_thck", p.cell_thck, cell_thck);
      UP(uint8_t, "col_ipl", p.col_ipl, col_ipl);
      v.x3 = a.get<double2>(s, "x3", (size_t)std::max(p.ncols, 1) * (v.nl + 1));
      v.eq3 = a.get<double>(s, "eq3", (size_t)std::max(p.ncells, 1) * 4 * v.nl);
      v.cell_omk = a.get<double>(s, "cell_omk", (size_t)std::max(p.ncells, 1) * (v.nl + 1));
      v.cell_om = a.get<double>(s, "cell_om", p.ncells);
      v.col_somega = a.get<double>(s, "col_somega", p.ncols);
      v.col_beff = a.get<double>(s, "col_beff", p.ncols);
      v.col_bt = a.get<double2>(s, "col_bt", p.ncols);
      upload(s, a.get<double>(s, "eq3_0", p.eq3_0.size()), p.eq3_0);
      upload(s, a.get<double2>(s, "bt0", p.col_bt0.size()), p.col_bt0);
    }
    v.badj = a.get<double>(s, "badj", 4 * np);
  }
  UP(int, "tile_start", p.tile_start, tile_start);
  UP(int, "tile_end", p.tile_end, tile_end);
  UP(int, "tile_inst", p.tile_inst, tile_inst);
  UP(int, "tile_ncols", p.tile_ncols, tile_ncols);
  UP(int, "tile_col0", p.tile_col0, tile_col0);
#undef UP
  v.A = a.get<double2>(s, "A", (v.sym ? 2 * 14 : 2 * 27) * np);
  v.x = a.get<double2>(s, "x", np);
  v.b = a.get<double2>(s, "b", np);
  v.r = a.get<double2>(s, "r", np);
  v.d0 = a.get<double2>(s, "d0", np);
  v.z = a.get<double2>(s, "z", np);
  v.q = a.get<double2>(s, "q", np);
  v.Az = a.get<double2>(s, "Az", np);
  v.Dinv = a.get<double2>(s, "Dinv", np);
  v.usav = a.get<double2>(s, "usav", np);
  // the hole slots of the node vectors stay zero
  for (double2* vec : {v.x, v.b, v.r, v.d0, v.z, v.q, v.Az, v.Dinv, v.usav})
    CK(cudaMemsetAsync(vec, 0, sizeof(double2) * np, s));
  bool any_sia = false;
  for (const auto& ip : p.inst) any_sia = any_sia || ip.precond == 2;
  v.sia_f = any_sia ? a.get<double2>(s, "sia_f", 3 * np) : nullptr;
  if (mixed && v.sym) {
    float4* blk = a.get<float4>(s, "A32", 16 * np);  // A32 then A32d: one L2 window
    v.A32 = blk;
    v.A32d = reinterpret_cast<double2*>(blk + 14 * np);
  }
  v.partials = a.get<double>(s, "partials", 3 * (size_t)std::max(p.ntiles, 1));
  v.tile_counter = a.get<unsigned>(s, "tile_counter", p.ninst);
  CK(cudaMemsetAsync(v.tile_counter, 0, sizeof(unsigned) * p.ninst, s));
  return v;
}

void init_state(cudaStream_t s, const DevView& v, const HostPlan& p, bool picard, bool pcg) {
  const int ninst = p.ninst;
  std::vector<InstState> st(ninst);
  int live = 0;
  for (int b = 0; b < ninst; ++b) {
    InstState& x = st[b];
    std::memset(&x, 0, sizeof(x));
    const bool empty = p.inst[b].node_end == p.inst[b].node_begin;
    // no active vertex at all: count_nonzeros_3d = 0, velocity zero
    // (glissade_velo_higher.F90:3191-3220)
    x.status = empty ? BP_ZERO_MATRIX : BP_OK;
    x.picard_active = (picard && !empty) ? 1 : 0;
    x.pcg_active = (pcg && !empty) ? 1 : 0;
    x.refine_active = x.pcg_active;
    x.pcg_iter = 1;
    x.rz = 1.0;
    x.rz_old = 1.0;
    x.err = -1.0;
    live += empty ? 0 : 1;
  }
  CK(cudaMemcpyAsync(v.st, st.data(), sizeof(InstState) * ninst, cudaMemcpyHostToDevice, s));
  Counters h{};
  h.picard_active = picard ? live : 0;
  h.pcg_active = pcg ? live : 0;
  h.refine_active = pcg ? live : 0;
  CK(cudaMemcpyAsync(v.cnt, &h, sizeof(h), cudaMemcpyHostToDevice, s));
  CK(cudaStreamSynchronize(s));  // st/h are host temporaries
}

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

// Launch with optional event timing.
template <typename F>
void L(bp_problem* P, int cat, F&& f) {
  Timing& T = P->timing;
  if (!T.on) {
    f();
    return;
  }
  const size_t i = T.cat.size();
  if (i >= T.pool.size()) {
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    T.pool.push_back({a, b});
  }
  CK(cudaEventRecord(T.pool[i].first, P->c->stream));
  f();
  CK(cudaEventRecord(T.pool[i].second, P->c->stream));
  T.cat.push_back(cat);
}

void collect_timing(bp_problem* P) {
  Timing& T = P->timing;
  if (!T.on) return;
  CK(cudaStreamSynchronize(P->c->stream));
  for (size_t i = 0; i < T.cat.size(); ++i) {
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, T.pool[i].first, T.pool[i].second));
    T.ms[T.cat[i]] += ms;
    T.n[T.cat[i]] += 1;
  }
  T.cat.clear();
}

enum { C_MV = 0, C_UPD = 1, C_CHECK = 2, C_MV32 = 3, C_UPD32 = 4, C_ASM1 = 5, C_ASM2 = 6, C_RHS = 7, C_OTHER = 8 };

// One PCG iteration n (standard or Chronopoulos-Gear), check included.
void enqueue_iteration(bp_problem* P, int variant, bool check) {
  const DevView& v = P->v;
  cudaStream_t s = P->c->stream;
  // mixed precision: the recurrence runs on through check iterations and
  // the check is the conditional refinement step
  const bool refine = v.A32 != nullptr;
  const bool upd_check = check && !refine;
  const int check_mode = refine ? MV_REFINE : MV_CHECK;
  if (variant == 3) {
    L(P, C_MV, [&] { launch_mv(MV_CG1, v, s); });
    L(P, C_UPD, [&] { launch_cg_update(upd_check, v, s); });
    if (check) L(P, C_CHECK, [&] { launch_mv(check_mode, v, s); });
  } else {
    L(P, C_MV, [&] { launch_mv(MV_STD_A, v, s); });
    L(P, C_UPD, [&] { launch_std_update(upd_check, v, s); });
    if (check) L(P, C_CHECK, [&] { launch_mv(check_mode, v, s); });
    L(P, C_UPD, [&] { launch_std_dir(v, s); });
  }
}

// A whole check chunk (ncheck iterations, the last one checks), captured
// once into a CUDA graph and replayed.
void enqueue_chunk(bp_problem* P, int variant, int ncheck) {
  cudaStream_t s = P->c->stream;
  if (P->use_graphs && !P->timing.on) {
    if (!P->chunk_graph) {
      cudaGraph_t g;
      CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      for (int j = 0; j < ncheck; ++j) enqueue_iteration(P, variant, j == ncheck - 1);
      CK(cudaStreamEndCapture(s, &g));
      CK(cudaGraphInstantiate(&P->chunk_graph, g, 0));
      CK(cudaGraphDestroy(g));
    }
    CK(cudaGraphLaunch(P->chunk_graph, s));
    return;
  }
  for (int j = 0; j < ncheck; ++j) enqueue_iteration(P, variant, j == ncheck - 1);
}

// Start of the PCG for the instances with pcg_active (after MV_INIT):
// d = z for the standard PCG; for Chronopoulos-Gear its first pass and the
// iterations before the first check (pcg:1304-1405).  Returns the number
// of the next iteration, which starts a check chunk.
int pcg_head(bp_problem* P) {
  const HostPlan& p = P->plan;
  const DevView& v = P->v;
  bp_ctx* c = P->c;
  const int variant = p.inst[0].variant;
  const int ncheck = std::max(1, p.inst[0].ncheck);
  int n = 1;
  if (variant == 3) {
    L(P, C_MV, [&] { launch_mv(MV_CG_FIRST, v, c->stream); });
    L(P, C_UPD, [&] { launch_cg_first_update(v, c->stream); });
    n = 2;
    while ((n - 1) % ncheck != 0) {
      enqueue_iteration(P, variant, (n % ncheck) == 0);
      ++n;
    }
  } else {
    L(P, C_UPD, [&] { launch_std_dir(v, c->stream); });  // d = z
  }
  return n;
}

// FP64 PCG for all instances with pcg_active, after MV_INIT: the head,
// then check chunks until the device counter shows no active instance (the
// host learns it one chunk late; the extra chunk's kernels find no active
// instance and return at once).
void run_pcg_fp64(bp_problem* P) {
  const HostPlan& p = P->plan;
  const DevView& v = P->v;
  bp_ctx* c = P->c;
  const int variant = p.inst[0].variant;
  const int ncheck = std::max(1, p.inst[0].ncheck);
  const int maxit = max_pcg_iters(p);
  int n = pcg_head(P);
  snapshot(c, v, 0);
  int chunk = 1;
  while (n <= maxit + 1) {
    enqueue_chunk(P, variant, ncheck);
    n += ncheck;
    snapshot(c, v, chunk & 1);
    if (wait_snapshot(c, (chunk - 1) & 1).pcg_active <= 0) break;
    ++chunk;
  }
  CK(cudaGetLastError());
}

// Linear solve of the assembled systems of all active instances.  With
// an FP32 matrix copy (mixed precision) the same kernels run the Krylov
// matvecs on it while every true residual stays FP64.
void linear_solve(bp_problem* P) {
  if (P->v.A32) L(P, C_OTHER, [&] { launch_make_a32(P->v, P->c->stream); });
  L(P, C_CHECK, [&] { launch_mv(MV_INIT, P->v, P->c->stream); });
  run_pcg_fp64(P);
}

// Autotuner: after the first assembly of a problem, time candidate launch
// shapes on the problem's own matrix and keep the fastest; results are
// cached per context by (size bucket, nz, storage, precision, PCG variant).
// Candidates time one warm-up and five timed launches.
//  * Residual kernels and the grid of the other tile kernels: the residual
//    matvec r = b - A x (k_resid<MV_INIT>, idempotent before the linear
//    solve, which recomputes it) for occupancy target 0 or 4 CTAs per SM
//    and grid one CTA per tile or 4 x SMs.
//  * Krylov matvecs, the solve's dominant kernel: the instance's own
//    kernel (k_cg_mv or k_std_mv on the FP32 or FP64 matrix) in a dry pass
//    (every tile, instance state untouched) for occupancy target 0, 4 or 6
//    and grid one CTA per tile or one wave of resident CTAs.  Its register
//    allocation, and so its occupancy, differs from the residual kernel's.
// BP_MV_CONFIG="minb,grid[,minb_k,grid_k]" fixes the choice (for sweeps);
// BP_TUNE_LOG=1 prints every candidate's time to stderr.
static float time_launches(bp_ctx* c, const std::function<void()>& launch) {
  launch();
  CK(cudaEventRecord(c->r0, c->stream));
  for (int i = 0; i < 5; ++i) launch();
  CK(cudaEventRecord(c->r1, c->stream));
  CK(cudaEventSynchronize(c->r1));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, c->r0, c->r1));
  return ms / 5.f;
}

void autotune(bp_problem* P) {
  bp_ctx* c = P->c;
  DevView& v = P->v;
  P->tuned = true;
  if (const char* e = std::getenv("BP_MV_CONFIG")) {
    int a[4] = {0, 0, 0, 0};
    const int n = std::sscanf(e, "%d,%d,%d,%d", &a[0], &a[1], &a[2], &a[3]);
    if (n == 2 || n == 4) {
      v.minb = a[0];
      v.grid_cap = a[1];
      v.minb_k = n == 4 ? a[2] : a[0];
      v.grid_k = n == 4 ? a[3] : a[1];
      return;
    }
  }
  const int variant = P->plan.inst.empty() ? 0 : P->plan.inst[0].variant;
  const auto key = std::make_tuple(P->plan.nnodes >> 14, P->plan.nz, v.sym, v.A32 ? 1 : 0, variant);
  auto it = c->tuned.find(key);
  if (it != c->tuned.end()) {
    v.minb = it->second[0];
    v.grid_cap = it->second[1];
    v.minb_k = it->second[2];
    v.grid_k = it->second[3];
    return;
  }
  const bool log = std::getenv("BP_TUNE_LOG") != nullptr;
  float best = 1e30f;
  int bm = 0, bg = 0;
  for (int mb : {0, 4})
    for (int g : {0, 4 * c->num_sms}) {
      if (g > 0 && g >= P->plan.ntiles) continue;  // same as one CTA per tile
      v.minb = mb;
      v.grid_cap = g;
      const float ms = time_launches(c, [&] { launch_mv(MV_INIT, v, c->stream); });
      if (log) std::fprintf(stderr, "autotune resid minb %d grid %d: %.2f us\n", mb, g, ms * 1e3f);
      if (ms < best) { best = ms; bm = mb; bg = g; }
    }
  v.minb = bm;
  v.grid_cap = bg;
  // the Krylov matvec on this storage (the FP32 copy is built here first:
  // the linear solve rebuilds it, so the dry pass reads a real matrix)
  if (v.A32) launch_make_a32(v, c->stream);
  const int mode = variant == 3 ? MV_CG1 : MV_STD_A;
  best = 1e30f;
  int km = 0, kg = 0;
  struct DryPass {  // the dry flag never outlives the timing, not even on an error
    DevView& v;
    explicit DryPass(DevView& w) : v(w) { v.dry = 1; }
    ~DryPass() { v.dry = 0; }
  };
  {
    const DryPass dry(v);
    for (int mb : {0, 4, 6, 8}) {
      const int res = krylov_resident_ctas(v, mode, mb);
      if (res <= 0) continue;
      for (int g : {0, res * c->num_sms}) {
        if (g > 0 && g >= P->plan.ntiles) continue;
        v.minb_k = mb;
        v.grid_k = g;
        const float ms = time_launches(c, [&] { launch_mv(mode, v, c->stream); });
        if (log)
          std::fprintf(stderr, "autotune krylov minb %d (%d CTAs/SM) grid %d: %.2f us\n", mb, res, g,
                       ms * 1e3f);
        if (ms < best) { best = ms; km = mb; kg = g; }
      }
    }
  }
  CK(cudaGetLastError());
  v.minb_k = km;
  v.grid_k = kg;
  c->tuned[key] = {bm, bg, km, kg};
}

// The Picard loop of glissade_velo_higher_solve on the device.
// Keeps the FP32 Krylov matrix of the mixed path (A32 with its FP64
// diagonal, one block) in L2 across the PCG iterations of a run.  Every
// matvec re-reads the whole block, and the update kernels stream about as
// many bytes of vectors in between, which would evict it.  The PCG
// kernels' launches carry an access-policy window that marks the block
// persisting, and for the run L2 is set aside for persisting lines up to
// the block's size (cudaLimitPersistingL2CacheSize, a limit of this
// process's CUDA context; at the end of the run the persisting lines are
// demoted and the previous limit restored).  Only when the block fits one
// window; BP_L2_PIN=0 turns it off.  These are cache hints: a failing call
// leaves the run as it is without them.
struct L2Pin {
  bp_problem* P;
  size_t old_limit = 0;
  bool set = false;
  explicit L2Pin(bp_problem* p) : P(p) {
    DevView& v = P->v;
    bp_ctx* c = P->c;
    v.l2_bytes = 0;
    const char* e = std::getenv("BP_L2_PIN");
    if (!v.A32 || (e && e[0] == '0') || c->l2_max_persist <= 0 || c->l2_max_window <= 0) return;
    // offsets 14..26 and the FP64 diagonal (entry 0 of A32 is not read)
    const size_t bytes = 15 * sizeof(float4) * (size_t)v.npad;
    if (bytes > (size_t)c->l2_max_window) return;
    const size_t aside = std::min(bytes, (size_t)c->l2_max_persist);
    if (cudaDeviceGetLimit(&old_limit, cudaLimitPersistingL2CacheSize) != cudaSuccess ||
        cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, aside) != cudaSuccess) {
      cudaGetLastError();
      return;
    }
    set = true;
    v.l2_base = v.A32 + v.npad;
    v.l2_bytes = bytes;
    v.l2_hit = (float)std::min(1.0, (double)aside / (double)bytes);
    if (std::getenv("BP_TUNE_LOG"))
      std::fprintf(stderr, "l2 pin: block %.1f MB, set aside %.1f MB (max %.1f MB, window max %.1f MB), hit %.3f\n",
                   bytes / 1e6, aside / 1e6, c->l2_max_persist / 1e6, c->l2_max_window / 1e6, v.l2_hit);
  }
  ~L2Pin() {
    if (!set) return;
    cudaStreamSynchronize(P->c->stream);
    cudaCtxResetPersistingL2Cache();
    cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, old_limit);
    cudaGetLastError();
  }
};

// One Picard iteration up to its linear solve: calcbeta for a sliding law,
// assembly (glissade_velo_higher.F90:2502-3119), the right-hand side, then
// (after the autotuner on the first assembly of a problem) the FP32 copy,
// the initial residual (:3191-3220) and the PCG head.
void picard_head(bp_problem* P, bool tune) {
  const HostPlan& p = P->plan;
  const DevView& v = P->v;
  cudaStream_t s = P->c->stream;
  L(P, C_OTHER, [&] { launch_picard_begin(v, s); });
  L(P, C_OTHER, [&] { launch_save_usav(v, s); });
  if (p.any_sliding) L(P, C_OTHER, [&] { launch_slide_beta(v, s); });
  L(P, C_ASM1, [&] { launch_asm_qp(v, s); });
  if (v.diva) L(P, C_ASM1, [&] { launch_diva_beta(v, s); });  // omega, beta_eff (:2742-2857)
  L(P, C_ASM2, [&] { launch_asm_rows(v, s); });
  L(P, C_RHS, [&] { launch_rhs(v, s); });
  if (v.sia_f) L(P, C_OTHER, [&] { launch_sia_factor(v, s); });
  if (tune && !P->tuned) autotune(P);
  if (P->v.A32) L(P, C_OTHER, [&] { launch_make_a32(P->v, s); });
  L(P, C_CHECK, [&] { launch_mv(MV_INIT, P->v, s); });
}

// The rest of a Picard iteration after its linear solve: DIVA's traction
// and 3-D velocity (:3658-3696), the Picard criterion (:3700-3727).
void picard_tail(bp_problem* P) {
  const DevView& v = P->v;
  cudaStream_t s = P->c->stream;
  if (v.diva) L(P, C_OTHER, [&] { launch_diva_velocity(v, s); });
  L(P, C_OTHER, [&] { launch_picard_check(v, s); });
}

int max_picard_iters(const HostPlan& p) {
  int m = 1;
  for (const auto& ip : p.inst) m = std::max(m, ip.maxiter_nonlinear);
  return m;
}

// The whole Picard loop as one CUDA graph that stays on the device:
//   reset -> WHILE (some instance in Picard, passes < cap) {
//     picard_head, PCG head, reset -> WHILE (some instance in PCG, chunks < cap) {
//       one check chunk of ncheck iterations; count }
//     picard_tail; count }
// The loop conditions are set by one-thread kernels (cudaGraphSetConditional)
// from the device counters the solve kernels keep, and each loop also stops
// after a pass cap above what the instances' own caps (maxiter_nonlinear,
// pcg_maxiters) allow, so the graph always ends.  The kernels are the host
// loop's, in its order, so the results are the same; the host waits once,
// after the graph.  Returns false where the graph cannot be built here
// (the host-driven loop then runs).
bool build_loop_graph(bp_problem* P, bool pdl) {
  const HostPlan& p = P->plan;
  const DevView& v = P->v;
  cudaStream_t s = P->c->stream;
  const int variant = p.inst[0].variant;
  const int ncheck = std::max(1, p.inst[0].ncheck);
  const int cap_picard = max_picard_iters(p) + 1;
  const int cap_chunks = max_pcg_iters(p) / ncheck + 3;
  if (!P->loop_iter) P->loop_iter = P->arena->get<int>(s, "loop_iter", 2);
  int* it = P->loop_iter;
  const auto mode = cudaStreamCaptureModeThreadLocal;
  cudaGraph_t g = nullptr;
  bool capturing = false;
  set_pdl(pdl);
  bool ok = false;
  try {
    CK(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle hP, hK;
    CK(cudaGraphConditionalHandleCreate(&hP, g, 0, 0));
    CK(cudaStreamBeginCaptureToGraph(s, g, nullptr, nullptr, 0, mode));
    capturing = true;
    launch_loop_cond(hP, v, true, it, cap_picard, true, s);
    CK(cudaStreamEndCapture(s, &g));
    capturing = false;
    cudaGraphNode_t start;
    size_t nn = 1;
    CK(cudaGraphGetNodes(g, &start, &nn));
    cudaGraphNodeParams wp = {};
    wp.type = cudaGraphNodeTypeConditional;
    wp.conditional.handle = hP;
    wp.conditional.type = cudaGraphCondTypeWhile;
    wp.conditional.size = 1;
    cudaGraphNode_t wP;
    CK(cudaGraphAddNode(&wP, g, &start, 1, &wp));
    cudaGraph_t bP = wp.conditional.phGraph_out[0];
    CK(cudaGraphConditionalHandleCreate(&hK, bP, 0, 0));
    // Picard body, up to the PCG loop
    CK(cudaStreamBeginCaptureToGraph(s, bP, nullptr, nullptr, 0, mode));
    capturing = true;
    picard_head(P, false);
    pcg_head(P);
    launch_loop_cond(hK, v, false, it + 1, cap_chunks, true, s);
    cudaStreamCaptureStatus cs;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    CK(cudaStreamGetCaptureInfo(s, &cs, nullptr, nullptr, &deps, &nd));
    std::vector<cudaGraphNode_t> last(deps, deps + nd);
    CK(cudaStreamEndCapture(s, &bP));
    capturing = false;
    cudaGraphNodeParams wk = {};
    wk.type = cudaGraphNodeTypeConditional;
    wk.conditional.handle = hK;
    wk.conditional.type = cudaGraphCondTypeWhile;
    wk.conditional.size = 1;
    cudaGraphNode_t wK;
    CK(cudaGraphAddNode(&wK, bP, last.data(), last.size(), &wk));
    cudaGraph_t bK = wk.conditional.phGraph_out[0];
    // PCG body: one check chunk
    CK(cudaStreamBeginCaptureToGraph(s, bK, nullptr, nullptr, 0, mode));
    capturing = true;
    for (int j = 0; j < ncheck; ++j) enqueue_iteration(P, variant, j == ncheck - 1);
    launch_loop_cond(hK, v, false, it + 1, cap_chunks, false, s);
    CK(cudaStreamEndCapture(s, &bK));
    capturing = false;
    // the rest of the Picard body, after the PCG loop
    CK(cudaStreamBeginCaptureToGraph(s, bP, &wK, nullptr, 1, mode));
    capturing = true;
    picard_tail(P);
    launch_loop_cond(hP, v, true, it, cap_picard, false, s);
    CK(cudaStreamEndCapture(s, &bP));
    capturing = false;
    ok = cudaGraphInstantiate(&P->loop_graph, g, 0) == cudaSuccess;
  } catch (const CudaError&) {
    ok = false;
  }
  if (capturing) {
    cudaGraph_t junk = nullptr;
    cudaStreamEndCapture(s, &junk);
  }
  set_pdl(true);
  if (g) cudaGraphDestroy(g);
  cudaGetLastError();  // a failed build leaves no sticky error: it only returned codes
  if (!ok) P->loop_graph = nullptr;
  return ok;
}

// BP_DEVICE_LOOP=0 keeps the host-driven Picard loop.
bool device_loop_wanted(const bp_problem* P) {
  const char* e = std::getenv("BP_DEVICE_LOOP");
  return P->use_graphs && !P->timing.on && P->loop_state >= 0 && !(e && e[0] == '0');
}

bool run_device_loop(bp_problem* P) {
  if (P->loop_state == 0) {
    // programmatic edges inside the loop bodies where the driver takes them
    const bool ok = build_loop_graph(P, true) || build_loop_graph(P, false);
    P->loop_state = ok ? 1 : -1;
    if (std::getenv("BP_TUNE_LOG"))
      std::fprintf(stderr, "device Picard loop: %s\n", ok ? "built" : "unavailable, host loop");
    if (!ok) return false;
  }
  CK(cudaGraphLaunch(P->loop_graph, P->c->stream));
  return true;
}

void run_picard(bp_problem* P) {
  const L2Pin pin(P);
  const DevView& v = P->v;
  bp_ctx* c = P->c;
  const int max_picard = max_picard_iters(P->plan);
  for (int it = 0; it < max_picard; ++it) {
    // the device loop takes over once the problem is tuned (the first run's
    // first assembly runs the autotuner on the host)
    if (P->tuned && device_loop_wanted(P) && run_device_loop(P)) break;
    picard_head(P, true);
    run_pcg_fp64(P);
    picard_tail(P);
    snapshot(c, v, 0);
    if (wait_snapshot(c, 0).picard_active <= 0) break;
  }
  CK(cudaGetLastError());
}

int final_status(const InstState& s) {
  if (s.status != BP_OK) return s.status;
  if (!s.picard_converged) return BP_WARN_PICARD_NOT_CONVERGED;
  if (!s.pcg_converged) return BP_WARN_PCG_NOT_CONVERGED;
  return BP_OK;
}

void fill_stats(const bp_problem* P, int b, bp_stats* st) {
  const InstState& s = P->state[b];
  std::memset(st, 0, sizeof(*st));
  st->status = final_status(s);
  st->picard_iters = s.picard_iter;
  st->pcg_iters_total = s.pcg_iters_total;
  st->pcg_iters_last = s.pcg_iters_last;
  st->refine_steps_total = s.refine_steps_total;
  st->converged = s.picard_converged;
  st->pcg_err_last = s.err;
  st->resid_velo = s.resid_velo;
  st->L2_norm = s.L2_norm;
  st->L2_norm_relative = s.L2_rel;
  st->ms_upload = P->ms_upload;
  st->h2d_bytes = P->h2d_bytes / std::max(1, P->plan.ninst);
  st->d2h_bytes = P->d2h_bytes / std::max(1, P->plan.ninst);
  st->ms_pcg = P->ms_solve;
  st->ms_total = P->ms_upload + P->ms_solve;
  if (P->timing.on)
    st->ms_assemble = (float)(P->timing.ms[C_ASM1] + P->timing.ms[C_ASM2] + P->timing.ms[C_RHS]);
}

int worst_status(const bp_problem* P) {
  int worst = BP_OK;
  for (const auto& s0 : P->state) {
    const int s = final_status(s0);
    const bool warn = s == BP_WARN_PCG_NOT_CONVERGED || s == BP_WARN_PICARD_NOT_CONVERGED || s == BP_ZERO_MATRIX;
    if (s == BP_OK) continue;
    if (worst == BP_OK || !warn) worst = s;
  }
  return worst;
}

bp_problem* problem_new(bp_ctx* c, Arena* arena, int n, const bp_inputs* in, std::string* err) {
  bp_problem* P = new bp_problem();
  P->c = c;
  P->arena = arena ? arena : &P->own;
  if (!build_plan(in, n, &P->plan, err)) {
    delete P;
    return nullptr;
  }
  P->mixed = P->plan.inst[0].precision == BP_MIXED;
  CK(cudaEventRecord(c->t0, c->stream));
  g_h2d = 0.0;
  P->v = make_view(*P->arena, c->stream, P->plan, true, P->mixed);
  P->h2d_bytes = g_h2d;
  P->x0 = P->arena->get<double2>(c->stream, "x0", P->plan.npad);
  CK(cudaMemsetAsync(P->x0, 0, sizeof(double2) * P->plan.npad, c->stream));
  if (P->plan.diva) {
    const size_t n3 = (size_t)std::max(P->plan.ncols, 1) * P->plan.nz_out;
    P->x3_0 = P->arena->get<double2>(c->stream, "x3_0", n3);
    CK(cudaMemsetAsync(P->x3_0, 0, sizeof(double2) * n3, c->stream));
    P->eq3_0 = P->arena->get<double>(c->stream, "eq3_0", P->plan.eq3_0.size());
    P->bt0 = P->arena->get<double2>(c->stream, "bt0", P->plan.col_bt0.size());
  }
  P->state.resize(n);
  return P;
}

void problem_free(bp_problem* P) {
  if (!P) return;
  if (P->chunk_graph) cudaGraphExecDestroy(P->chunk_graph);
  if (P->inner_graph) cudaGraphExecDestroy(P->inner_graph);
  if (P->loop_graph) cudaGraphExecDestroy(P->loop_graph);
  P->timing.destroy();
  P->own.release();
  delete P;
}

void problem_set_guess(bp_problem* P, double* const* uvel, double* const* vvel) {
  std::vector<double2> x(P->plan.npad, double2{0.0, 0.0});
  std::vector<int> learned;
  for (int b = 0; b < P->plan.ninst; ++b) {
    if (P->plan.guess_mode[b] == BP_GUESS_LEARNED) learned.push_back(b);
    else gather_velocity(P->plan, b, uvel[b], vvel[b], x.data());
  }
  CK(cudaMemcpyAsync(P->x0, x.data(), sizeof(double2) * P->plan.npad, cudaMemcpyHostToDevice, P->c->stream));
  P->h2d_bytes += sizeof(double2) * (double)P->plan.nnodes;
  if (!learned.empty()) {  // the network's guess straight into x0, on the device
    if (!P->c->net) throw GuessError{"guess_mode = BP_GUESS_LEARNED needs bp_guess_load"};
    if (guess_net_run(P->c->net, P->plan, P->v, learned, P->x0, P->c->stream, &P->c->net_launches) != BP_OK)
      throw GuessError{"the learned guess failed"};
  }
  std::vector<double2> x3;
  if (P->plan.diva && P->plan.ncols > 0) {  // the first iteration's sliding law reads its bed level
    x3.assign((size_t)P->plan.ncols * P->plan.nz_out, double2{0.0, 0.0});
    for (int b = 0; b < P->plan.ninst; ++b) gather_velocity_3d(P->plan, b, uvel[b], vvel[b], x3.data());
    CK(cudaMemcpyAsync(P->x3_0, x3.data(), sizeof(double2) * x3.size(), cudaMemcpyHostToDevice, P->c->stream));
    P->h2d_bytes += sizeof(double2) * (double)x3.size();
  }
  CK(cudaStreamSynchronize(P->c->stream));
}

void problem_run(bp_problem* P) {
  bp_ctx* c = P->c;
  if (P->timing.on) {
    if (!P->mv_nodes_dev) P->mv_nodes_dev = P->arena->get<unsigned long long>(c->stream, "mv_nodes", 2);
    CK(cudaMemsetAsync(P->mv_nodes_dev, 0, 2 * sizeof(unsigned long long), c->stream));
    P->v.mv_nodes = P->mv_nodes_dev;
  } else {
    P->v.mv_nodes = nullptr;
  }
  CK(cudaEventRecord(c->t1, c->stream));
  CK(cudaMemcpyAsync(P->v.x, P->x0, sizeof(double2) * P->plan.npad, cudaMemcpyDeviceToDevice, c->stream));
  if (P->v.diva && P->plan.ncols > 0) {
    CK(cudaMemcpyAsync(P->v.x3, P->x3_0, sizeof(double2) * (size_t)P->plan.ncols * P->plan.nz_out,
                       cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(P->v.col_bt, P->bt0, sizeof(double2) * P->plan.col_bt0.size(), cudaMemcpyDeviceToDevice,
                       c->stream));
    if (!P->plan.eq3_0.empty())
      CK(cudaMemcpyAsync(P->v.eq3, P->eq3_0, sizeof(double) * P->plan.eq3_0.size(), cudaMemcpyDeviceToDevice,
                         c->stream));
  }
  init_state(c->stream, P->v, P->plan, true, false);
  run_picard(P);
  if (P->v.l1l2) launch_l1l2_velocity(P->v, c->stream);  // compute_3d_velocity_L1L2 (:3773-3801)
  CK(cudaEventRecord(c->t2, c->stream));
  CK(cudaMemcpyAsync(P->state.data(), P->v.st, sizeof(InstState) * P->plan.ninst,
                     cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  collect_timing(P);
  if (P->v.mv_nodes) {
    CK(cudaMemcpy(P->mv_nodes, P->mv_nodes_dev, sizeof(P->mv_nodes), cudaMemcpyDeviceToHost));
    P->v.mv_nodes = nullptr;
  }
  cudaEventElapsedTime(&P->ms_solve, c->t1, c->t2);
}

void problem_get(bp_problem* P, double* const* uvel, double* const* vvel, double* const* efvs) {
  const HostPlan& p = P->plan;
  // L1L2 and DIVA: the 3-D velocity, else the solution vector
  const bool v3 = p.l1l2 || p.diva;
  const size_t nx = v3 ? (size_t)p.ncols * p.nz_out : (size_t)p.npad;
  std::vector<double2> x(std::max<size_t>(nx, 1));
  if (nx > 0)
    CK(cudaMemcpyAsync(x.data(), v3 ? P->v.x3 : P->v.x, sizeof(double2) * nx, cudaMemcpyDeviceToHost,
                       P->c->stream));
  std::vector<double2> x2, bt;  // DIVA: the mean velocity and the traction
  if (p.diva && p.ncols > 0) {  // the mean velocity in node order (col_node), the traction per column
    x2.resize(p.npad);
    bt.resize(p.ncols);
    CK(cudaMemcpyAsync(x2.data(), P->v.x, sizeof(double2) * p.npad, cudaMemcpyDeviceToHost, P->c->stream));
    CK(cudaMemcpyAsync(bt.data(), P->v.col_bt, sizeof(double2) * p.ncols, cudaMemcpyDeviceToHost, P->c->stream));
  }
  std::vector<double> ef;
  if (efvs) {
    ef.resize(std::max(p.nefvs, 1));
    if (p.nefvs > 0)
      CK(cudaMemcpyAsync(ef.data(), P->v.efvs, sizeof(double) * p.nefvs, cudaMemcpyDeviceToHost, P->c->stream));
  }
  CK(cudaStreamSynchronize(P->c->stream));
  P->d2h_bytes = sizeof(double2) * (double)(v3 ? nx : (size_t)p.nnodes) +
                 (efvs ? sizeof(double) * (double)p.nefvs : 0.0) + sizeof(double2) * 2.0 * (double)bt.size();
  for (int b = 0; b < p.ninst; ++b) {
    if (uvel && vvel) {
      if (v3) scatter_velocity_3d(p, b, x.data(), uvel[b], vvel[b]);
      else scatter_velocity(p, b, x.data(), uvel[b], vvel[b]);
    }
    if (p.diva) scatter_diva(p, b, x2.empty() ? nullptr : x2.data(), bt.empty() ? nullptr : bt.data());
    if (efvs && efvs[b]) scatter_efvs(p, b, ef.data(), efvs[b]);
  }
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
    CK(cudaEventCreate(&c->r0));
    CK(cudaEventCreate(&c->r1));
    CK(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device));
    if (cudaDeviceGetAttribute(&c->l2_max_persist, cudaDevAttrMaxPersistingL2CacheSize, device) != cudaSuccess ||
        cudaDeviceGetAttribute(&c->l2_max_window, cudaDevAttrMaxAccessPolicyWindowSize, device) != cudaSuccess) {
      c->l2_max_persist = c->l2_max_window = 0;
      cudaGetLastError();
    }
    CK(bp::upload_ref_tables());
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
  c->arena.release();
  if (c->net) guess_net_free(c->net);
  if (c->h_cnt) cudaFreeHost(c->h_cnt);
  for (auto& e : c->ev)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : {c->t0, c->t1, c->t2, c->t3, c->r0, c->r1})
    if (e) cudaEventDestroy(e);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return BP_OK;
}

const char* bp_last_error(const bp_ctx* c) { return c ? c->err.c_str() : "no context"; }

#define GUARD_BEGIN(ctx)            \
  bp_ctx* c_ = (ctx);               \
  if (!c_) return BP_ERR_ARGS;      \
  c_->err.clear();                  \
  try {                             \
    CK(cudaSetDevice(c_->device));
#define GUARD_END                                                      \
  }                                                                    \
  catch (const CudaError& e) {                                         \
    c_->err = std::string(e.what) + ": " + cudaGetErrorString(e.e);    \
    return BP_ERR_CUDA;                                                \
  }                                                                    \
  catch (const GuessError& e) {                                        \
    c_->err = e.what;                                                  \
    return BP_ERR_ARGS;                                                \
  }                                                                    \
  return BP_ERR_CUDA;

int bp_problem_create(bp_ctx* c, int n, const bp_inputs* in, bp_problem** out) {
  GUARD_BEGIN(c)
  if (!out || n < 1 || !in) return BP_ERR_ARGS;
  *out = nullptr;
  std::string err;
  bp_problem* P = problem_new(c, nullptr, n, in, &err);
  if (!P) {
    c->err = err;
    return BP_ERR_ARGS;
  }
  CK(cudaEventRecord(c->t3, c->stream));
  CK(cudaEventSynchronize(c->t3));
  cudaEventElapsedTime(&P->ms_upload, c->t0, c->t3);
  *out = P;
  return BP_OK;
  GUARD_END
}

int bp_problem_set_guess(bp_problem* P, double* const* uvel, double* const* vvel) {
  if (!P) return BP_ERR_ARGS;
  GUARD_BEGIN(P->c)
  for (int b = 0; b < P->plan.ninst; ++b)
    if (P->plan.guess_mode[b] != BP_GUESS_LEARNED && (!uvel || !vvel || !uvel[b] || !vvel[b])) return BP_ERR_ARGS;
  problem_set_guess(P, uvel, vvel);
  CK(cudaStreamSynchronize(P->c->stream));
  return BP_OK;
  GUARD_END
}

int bp_problem_get_guess(bp_problem* P, double* const* uvel, double* const* vvel) {
  if (!P) return BP_ERR_ARGS;
  GUARD_BEGIN(P->c)
  if (!uvel || !vvel || P->plan.l1l2 || P->plan.diva) return BP_ERR_ARGS;
  std::vector<double2> x(P->plan.npad);
  CK(cudaMemcpyAsync(x.data(), P->x0, sizeof(double2) * P->plan.npad, cudaMemcpyDeviceToHost, P->c->stream));
  CK(cudaStreamSynchronize(P->c->stream));
  for (int b = 0; b < P->plan.ninst; ++b) scatter_velocity(P->plan, b, x.data(), uvel[b], vvel[b]);
  return BP_OK;
  GUARD_END
}

int bp_guess_load(bp_ctx* c, const char* path) {
  GUARD_BEGIN(c)
  if (!path) return BP_ERR_ARGS;
  std::string err;
  bp::GuessNet* N = guess_net_load(path, &err);
  if (!N) {
    c->err = err;
    return BP_ERR_ARGS;
  }
  if (c->net) guess_net_free(c->net);
  c->net = N;
  return BP_OK;
  GUARD_END
}

int bp_guess_launches(bp_ctx* c) { return c ? c->net_launches : 0; }

int bp_problem_run(bp_problem* P, bp_stats* stats) {
  if (!P) return BP_ERR_ARGS;
  GUARD_BEGIN(P->c)
  problem_run(P);
  if (stats)
    for (int b = 0; b < P->plan.ninst; ++b) fill_stats(P, b, &stats[b]);
  return worst_status(P);
  GUARD_END
}

int bp_problem_get(bp_problem* P, double* const* uvel, double* const* vvel, double* const* efvs) {
  if (!P) return BP_ERR_ARGS;
  GUARD_BEGIN(P->c)
  problem_get(P, uvel, vvel, efvs);
  return BP_OK;
  GUARD_END
}

int bp_problem_diagnostics(bp_problem* P, int which_bfric, double* const* tau_xz,
                           double* const* tau_yz, double* const* tau_xx,
                           double* const* tau_yy, double* const* tau_xy,
                           double* const* tau_eff, double* const* bfricflx) {
  if (!P || (which_bfric != 0 && which_bfric != 1)) return BP_ERR_ARGS;
  GUARD_BEGIN(P->c)
  const HostPlan& p = P->plan;
  bp_ctx* c = P->c;
  double* const* outs[6] = {tau_xz, tau_yz, tau_xx, tau_yy, tau_xy, tau_eff};
  bool want_tau = false;
  for (auto o : outs) want_tau = want_tau || o;
  if (!p.ncells) return BP_ERR_ARGS;  // matrix-level problems have no elements
  // 2-D solves: the 3-D elements over the model's levels with the 3-D
  // velocity (L1L2, DIVA: the one the solve formed; shallow-shelf: its
  // solution on every level) and, for the shallow-shelf stresses, the flow
  // factor of each layer; DIVA's bed-face corners take beta_internal again
  // (the loop left beta_eff there)
  double2* x3 = P->v.x3;
  const double* fl = nullptr;
  if (p.solve2d && !p.l1l2 && !p.diva) {
    x3 = P->arena->get<double2>(c->stream, "diag_x3", (size_t)std::max(p.ncols, 1) * p.nz_out);
    launch_levels_from_2d(P->v, x3, p.nz_out, c->stream);
    double* f = P->arena->get<double>(c->stream, "diag_flwafact", p.flwafact_layers.size());
    upload(c->stream, f, p.flwafact_layers);
    fl = f;
  }
  if (p.diva) {
    if (p.any_sliding) launch_corner_beta(P->v, c->stream);
    else upload(c->stream, P->v.cell_beta, p.cell_beta);
  }
  int* cn3 = nullptr;
  if (p.solve2d) {  // x3 is [ncols][nz_out]
    std::vector<int> h3(std::max(p.ncols, 1));
    for (int c = 0; c < p.ncols; ++c) h3[c] = c * p.nz_out;
    cn3 = P->arena->get<int>(c->stream, "diag_col_node", h3.size());
    upload(c->stream, cn3, h3);
  }
  const DevView dv = diagnostics_view(P->v, p, x3, fl, cn3);
  const size_t ne = (size_t)diagnostic_elements(p), nb = (size_t)std::max(p.ncells, p.ncols);
  double* d = P->arena->get<double>(c->stream, "diagnostics", (want_tau ? 6 * ne : 0) + nb);
  double* d_tau = want_tau ? d : nullptr;
  double* d_bf = bfricflx ? d + (want_tau ? 6 * ne : 0) : nullptr;
  launch_diagnostics(dv, which_bfric, d_tau, d_bf, c->stream);
  std::vector<double> tau(d_tau ? 6 * ne : 0), bf(d_bf ? nb : 0);
  if (d_tau) CK(cudaMemcpyAsync(tau.data(), d_tau, sizeof(double) * tau.size(), cudaMemcpyDeviceToHost, c->stream));
  if (d_bf) CK(cudaMemcpyAsync(bf.data(), d_bf, sizeof(double) * bf.size(), cudaMemcpyDeviceToHost, c->stream));
  std::vector<InstState> st(p.ninst);
  CK(cudaMemcpyAsync(st.data(), P->v.st, sizeof(InstState) * p.ninst, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaGetLastError());
  int rc = BP_OK;
  for (int b = 0; b < p.ninst; ++b) {
    if (st[b].status == BP_ERR_SINGULAR_JAC) rc = BP_ERR_SINGULAR_JAC;
    if (d_tau) {
      double* o[6];
      for (int f = 0; f < 6; ++f) o[f] = outs[f] ? outs[f][b] : nullptr;
      scatter_elements(p, b, tau.data(), 6, o);
    }
    if (d_bf) scatter_bfric(p, b, which_bfric, bf.data(), bfricflx[b]);
  }
  return rc;
  GUARD_END
}

int bp_problem_destroy(bp_problem* P) {
  if (!P) return BP_OK;
  cudaSetDevice(P->c->device);
  cudaStreamSynchronize(P->c->stream);
  problem_free(P);
  return BP_OK;
}

int bp_timer_start(bp_ctx* c) {
  GUARD_BEGIN(c)
  CK(cudaEventRecord(c->r0, c->stream));
  return BP_OK;
  GUARD_END
}

int bp_timer_stop(bp_ctx* c, float* ms) {
  GUARD_BEGIN(c)
  CK(cudaEventRecord(c->r1, c->stream));
  CK(cudaEventSynchronize(c->r1));
  float t = 0.f;
  CK(cudaEventElapsedTime(&t, c->r0, c->r1));
  if (ms) *ms = t;
  return BP_OK;
  GUARD_END
}

int bp_problem_timing(bp_problem* P, int enable) {
  if (!P) return BP_ERR_ARGS;
  P->timing.on = enable != 0;
  P->timing.reset();
  return BP_OK;
}

int bp_problem_kernel_times(bp_problem* P, double* ms, int* launches) {
  if (!P) return BP_ERR_ARGS;
  for (int i = 0; i < BP_NUM_KERNEL_CATEGORIES; ++i) {
    if (ms) ms[i] = P->timing.ms[i];
    if (launches) launches[i] = P->timing.n[i];
  }
  return BP_OK;
}

int bp_problem_tune_mv(bp_problem* P, int store, int minb, int grid, int reps, float* ms) {
  if (!P) return BP_ERR_ARGS;
  GUARD_BEGIN(P->c)
  bp_ctx* c = P->c;
  if (store == 2 && P->v.sym && !P->v.A32) {
    float4* blk = P->arena->get<float4>(c->stream, "A32", 16 * (size_t)P->plan.npad);
    P->v.A32 = blk;
    P->v.A32d = reinterpret_cast<double2*>(blk + 14 * (size_t)P->plan.npad);
    launch_make_a32(P->v, c->stream);
  }
  if (launch_tune_mv(store, minb, grid, P->v, c->stream) != 0) return BP_ERR_ARGS;  // warm
  CK(cudaEventRecord(c->r0, c->stream));
  for (int i = 0; i < reps; ++i) launch_tune_mv(store, minb, grid, P->v, c->stream);
  CK(cudaEventRecord(c->r1, c->stream));
  CK(cudaEventSynchronize(c->r1));
  CK(cudaGetLastError());
  float t = 0.f;
  CK(cudaEventElapsedTime(&t, c->r0, c->r1));
  if (ms) *ms = t / std::max(1, reps);
  if (store == 2 && !P->mixed) {  // keep the FP64 path unchanged
    P->v.A32 = nullptr;
    P->v.A32d = nullptr;
  }
  return BP_OK;
  GUARD_END
}

int bp_problem_mv_nodes(bp_problem* P, double* fp64_nodes, double* fp32_nodes, int* minb, int* grid) {
  if (!P) return BP_ERR_ARGS;
  if (fp64_nodes) *fp64_nodes = (double)P->mv_nodes[0];
  if (fp32_nodes) *fp32_nodes = (double)P->mv_nodes[1];
  if (minb) *minb = P->v.minb_k;
  if (grid) *grid = P->v.grid_k;
  return BP_OK;
}

int bp_problem_info(bp_problem* P, long* nodes, long* cols, long* elems, double* mvb64,
                    double* mvb32) {
  if (!P) return BP_ERR_ARGS;
  const double N = (double)P->plan.nnodes;
  if (nodes) *nodes = P->plan.nnodes;
  if (cols) *cols = P->plan.ncols;
  if (elems) *elems = P->plan.nelem;
  // algorithmic bytes of one Krylov matvec launch per node: the stored
  // matrix once -- FP64 half storage 14 offsets x 2 rows x (u, v) doubles =
  // 448 B (full rows 864 B); FP32 half storage 13 offsets x 4 floats +
  // the FP64 diagonal block 32 B = 240 B; the lower half is re-read from
  // the neighbours' rows, in cache -- plus the vectors: the source read and
  // the result written (standard PCG: d, q), and for Chronopoulos-Gear r
  // read for the fused dots (z, r, Az)
  const bool cg = P->plan.inst[0].variant == 3;
  const double vec = (cg ? 3.0 : 2.0) * 16.0;
  if (mvb64) *mvb64 = N * ((P->v.sym ? 448.0 : 864.0) + vec);
  if (mvb32) *mvb32 = N * (240.0 + vec);
  return BP_OK;
}

int bp_batch_solve(bp_ctx* c, int n, const bp_inputs* in, double* const* uvel,
                   double* const* vvel, double* const* efvs, bp_stats* stats) {
  GUARD_BEGIN(c)
  if (n < 1 || !in || !uvel || !vvel) return BP_ERR_ARGS;
  std::string err;
  bp_problem* P = problem_new(c, &c->arena, n, in, &err);
  if (!P) {
    c->err = err;
    return BP_ERR_ARGS;
  }
  int rc = BP_OK;
  try {
    problem_set_guess(P, uvel, vvel);
    CK(cudaEventRecord(c->t3, c->stream));
    CK(cudaEventSynchronize(c->t3));
    cudaEventElapsedTime(&P->ms_upload, c->t0, c->t3);
    problem_run(P);
    problem_get(P, uvel, vvel, efvs);
    if (stats)
      for (int b = 0; b < n; ++b) fill_stats(P, b, &stats[b]);
    rc = worst_status(P);
  } catch (...) {
    problem_free(P);
    throw;
  }
  problem_free(P);
  return rc;
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
  GUARD_BEGIN(c)
  if (!active_vertex || !Auu || !Auv || !Avu || !Avv || !bu || !bv || !xu || !xv)
    return BP_ERR_ARGS;
  if (precond < 0 || precond > 2) {
    c->err = "bp_pcg: precond must be 0, 1 or 2";
    return BP_ERR_ARGS;
  }
  if (precision != BP_FP64) {
    c->err = "bp_pcg: an external matrix is solved in FP64 (precision 0)";
    return BP_ERR_ARGS;
  }
  bp_problem P;
  P.c = c;
  P.arena = &c->arena;
  std::string e;
  if (!build_column_plan(nx, ny, nz, periodic, active_vertex, &P.plan, &e)) {
    c->err = e;
    return BP_ERR_ARGS;
  }
  InstParams& ip = P.plan.inst[0];
  ip.precond = precond;
  ip.variant = variant == 3 ? 3 : 2;
  ip.pcg_tol = tol;
  ip.pcg_maxiters = maxiters;
  ip.ncheck = ncheck > 0 ? ncheck : 5;
  ip.precision = precision;
  ip.inner_tol = 1.0e-4;
  P.mixed = false;
  P.use_graphs = false;
  P.v = make_view(*P.arena, c->stream, P.plan, false, P.mixed);
  const DevView& v = P.v;
  std::vector<double2> A(2 * 27 * (size_t)P.plan.npad);
  gather_matrix(P.plan, Auu, Auv, Avu, Avv, A.data());
  CK(cudaMemcpyAsync(v.A, A.data(), sizeof(double2) * A.size(), cudaMemcpyHostToDevice, c->stream));
  std::vector<double2> x(P.plan.npad, double2{0, 0}), b(P.plan.npad, double2{0, 0});
  gather_velocity(P.plan, 0, xu, xv, x.data());
  gather_velocity(P.plan, 0, bu, bv, b.data());
  CK(cudaMemcpyAsync(v.x, x.data(), sizeof(double2) * P.plan.npad, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(v.b, b.data(), sizeof(double2) * P.plan.npad, cudaMemcpyHostToDevice, c->stream));
  init_state(c->stream, v, P.plan, false, true);
  launch_sia_factor(v, c->stream);
  launch_dinv(v, precond, c->stream);
  launch_bb(v, c->stream);
  linear_solve(&P);
  CK(cudaMemcpyAsync(x.data(), v.x, sizeof(double2) * P.plan.npad, cudaMemcpyDeviceToHost, c->stream));
  InstState st;
  CK(cudaMemcpyAsync(&st, v.st, sizeof(st), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaGetLastError());
  scatter_velocity(P.plan, 0, x.data(), xu, xv);
  if (err) *err = st.err;
  if (niters) *niters = P.mixed ? st.pcg_iters_total : st.pcg_iters_last;
  if (st.status != BP_OK) return st.status;
  return st.pcg_converged ? BP_OK : BP_WARN_PCG_NOT_CONVERGED;
  GUARD_END
}

int bp_matvec(bp_ctx* c, int nx, int ny, int nz, int periodic,
              const int* active_vertex, const double* Auu, const double* Auv,
              const double* Avu, const double* Avv, const double* xu,
              const double* xv, double* yu, double* yv) {
  GUARD_BEGIN(c)
  if (!active_vertex || !Auu || !Auv || !Avu || !Avv || !xu || !xv || !yu || !yv)
    return BP_ERR_ARGS;
  HostPlan p;
  std::string e;
  if (!build_column_plan(nx, ny, nz, periodic, active_vertex, &p, &e)) {
    c->err = e;
    return BP_ERR_ARGS;
  }
  DevView v = make_view(c->arena, c->stream, p, false, false);
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
  GUARD_BEGIN(c)
  if (!in || !uvel || !vvel) return BP_ERR_ARGS;
  HostPlan p;
  std::string e;
  if (!build_plan(in, 1, &p, &e)) {
    c->err = e;
    return BP_ERR_ARGS;
  }
  if (p.solve2d) {  // the 2-D system has the 9-entry reference layout, not this one
    c->err = "bp_assemble: 3-D Blatter-Pattyn systems only";
    return BP_ERR_ARGS;
  }
  DevView v = make_view(c->arena, c->stream, p, true, false);
  std::vector<double2> x(p.npad, double2{0, 0});
  gather_velocity(p, 0, uvel, vvel, x.data());
  CK(cudaMemcpyAsync(v.x, x.data(), sizeof(double2) * p.npad, cudaMemcpyHostToDevice, c->stream));
  init_state(c->stream, v, p, true, false);
  launch_picard_begin(v, c->stream);
  if (p.any_sliding) launch_slide_beta(v, c->stream);
  launch_asm_qp(v, c->stream);
  launch_asm_rows(v, c->stream);
  launch_rhs(v, c->stream);
  std::vector<double2> A((v.sym ? 2 * 14 : 2 * 27) * (size_t)p.npad), b(p.npad);
  std::vector<double> ef(std::max(p.nelem, 1));
  CK(cudaMemcpyAsync(A.data(), v.A, sizeof(double2) * A.size(), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(b.data(), v.b, sizeof(double2) * p.npad, cudaMemcpyDeviceToHost, c->stream));
  if (p.nelem > 0)
    CK(cudaMemcpyAsync(ef.data(), v.efvs, sizeof(double) * p.nelem, cudaMemcpyDeviceToHost, c->stream));
  InstState st;
  CK(cudaMemcpyAsync(&st, v.st, sizeof(st), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaGetLastError());
  if (v.sym) scatter_matrix_sym(p, A.data(), Auu, Auv, Avu, Avv);
  else scatter_matrix(p, A.data(), Auu, Auv, Avu, Avv);
  const size_t tot = (size_t)in->nz * (in->nx - 1) * (in->ny - 1);
  if (bu) std::memset(bu, 0, sizeof(double) * tot);
  if (bv) std::memset(bv, 0, sizeof(double) * tot);
  scatter_vector(p, 0, b.data(), bu, bv);
  if (efvs) scatter_efvs(p, 0, ef.data(), efvs);
  return st.status;
  GUARD_END
}

}  // extern "C"
