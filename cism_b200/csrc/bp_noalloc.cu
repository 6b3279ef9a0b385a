// bp_noalloc.cu -- residual and norms without any device allocation.
//
// bp_residual_noalloc computes resid = A x - b on the locally owned active
// rows of a system held by the caller in device memory, in the reference's
// own layout (matrix blocks (27,nz,nx-1,ny-1), vectors (nz,nx-1,ny-1), halo
// included and already halo-consistent), plus |A x - b|, |b| and their
// ratio.  It is the allocation-free variant of the residual kernel of the
// solver (k_mv<MV_INIT>): its only scratch -- one partial sum pair per
// block and the ticket that elects the block doing the final sum -- lives in
// the file-scope array below instead of in memory from cudaMalloc.
//
// Who needs it: a host model that owns all device memory itself (a fixed
// pool or budget set up once) or that must not trigger the implicit
// device-wide synchronisation of cudaMalloc/cudaFree in the middle of a
// time step can call this with its own buffers and nothing else.
//
// Limits and sharing: at most kNaMaxRows = 16,777,216 rows (nz*(nx-1)*(ny-1));
// larger systems are rejected with BP_ERR_ARGS.  The array is global to the
// process and to each device, and every call reuses it: two calls whose
// work overlaps on the GPU (different streams, or different host threads on
// one device) race on the partial sums and give wrong norms.  Serialise
// them.  The first call on a device (and the first after the device's
// context was torn down and made again, e.g. by cudaDeviceReset) looks up
// the array's device address (cudaGetSymbolAddress); make that call before
// any stream capture.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "bp_b200.h"

namespace {

constexpr int kNaBlock = 256;
constexpr int kNaMaxBlocks = 65536;
constexpr long kNaMaxRows = (long)kNaBlock * kNaMaxBlocks;
constexpr int kNaMaxDevices = 64;

struct NaScratch {
  double partial[2 * kNaMaxBlocks];  // per block: sum (Ax-b)^2, sum b^2
  unsigned ticket;                   // blocks finished (zeroed before each launch)
  unsigned pad[63];
};

// 1 MiB + 256 B on every device that loads the library, held until exit.
static __device__ __align__(256) NaScratch g_na_scratch;

std::mutex g_na_mutex;
NaScratch* g_na_ptr[kNaMaxDevices] = {nullptr};

__global__ void __launch_bounds__(kNaBlock)
k_resid_ref_layout(int nx, int ny, int nz, int periodic, const int* __restrict__ active_vertex,
                   const double* __restrict__ Auu, const double* __restrict__ Auv,
                   const double* __restrict__ Avu, const double* __restrict__ Avv,
                   const double* __restrict__ xu, const double* __restrict__ xv,
                   const double* __restrict__ bu, const double* __restrict__ bv,
                   double* __restrict__ ru, double* __restrict__ rv, double* __restrict__ norms,
                   NaScratch* S) {
  const int V = nx - 1, W = ny - 1;
  const long rows = (long)nz * V * W;
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  double s_r = 0.0, s_b = 0.0;
  if (t < rows) {
    const int k = (int)(t % nz);
    const long c = t / nz;
    const int i = (int)(c % V) + 1, j = (int)(c / V) + 1;  // 1-based vertex indices
    const int ilo = periodic ? 3 : 2, jlo = periodic ? 3 : 2;
    const bool owned = i >= ilo && i <= nx - 2 && j >= jlo && j <= ny - 2;
    double yu = 0.0, yv = 0.0;
    if (owned && active_vertex[c]) {
      // matvec_multiply_structured_3d order: kA, jA, iA; neighbours are
      // read directly at (halo) indices, as the reference does
      for (int kA = -1; kA <= 1; ++kA) {
        if (k + kA < 0 || k + kA >= nz) continue;
        for (int jA = -1; jA <= 1; ++jA)
          for (int iA = -1; iA <= 1; ++iA) {
            const int m = (iA + 1) + 3 * (jA + 1) + 9 * (kA + 1);
            const long a = t * 27 + m;
            const long x = ((long)(j + jA - 1) * V + (i + iA - 1)) * nz + (k + kA);
            yu = yu + Auu[a] * xu[x] + Auv[a] * xv[x];
            yv = yv + Avu[a] * xu[x] + Avv[a] * xv[x];
          }
      }
      yu -= bu[t];
      yv -= bv[t];
      s_r = yu * yu + yv * yv;
      s_b = bu[t] * bu[t] + bv[t] * bv[t];
    }
    ru[t] = yu;
    rv[t] = yv;
  }
  // block sums (fixed tree), one partial pair per block
  __shared__ double sh[2][kNaBlock / 32];
  for (int o = 16; o > 0; o >>= 1) {
    s_r += __shfl_xor_sync(0xffffffffu, s_r, o);
    s_b += __shfl_xor_sync(0xffffffffu, s_b, o);
  }
  if ((threadIdx.x & 31) == 0) {
    sh[0][threadIdx.x >> 5] = s_r;
    sh[1][threadIdx.x >> 5] = s_b;
  }
  __syncthreads();
  __shared__ int last;
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int w = 0; w < kNaBlock / 32; ++w) { a += sh[0][w]; b += sh[1][w]; }
    S->partial[2 * blockIdx.x] = a;
    S->partial[2 * blockIdx.x + 1] = b;
    __threadfence();
    last = (atomicAdd(&S->ticket, 1u) == gridDim.x - 1) ? 1 : 0;
  }
  __syncthreads();
  if (!last) return;
  // the last block sums every partial in block order
  __threadfence();
  double a = 0.0, b = 0.0;
  for (unsigned q = threadIdx.x; q < gridDim.x; q += blockDim.x) {
    a += __ldcg(&S->partial[2 * q]);
    b += __ldcg(&S->partial[2 * q + 1]);
  }
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  if ((threadIdx.x & 31) == 0) {
    sh[0][threadIdx.x >> 5] = a;
    sh[1][threadIdx.x >> 5] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double ta = 0.0, tb = 0.0;
    for (int w = 0; w < kNaBlock / 32; ++w) { ta += sh[0][w]; tb += sh[1][w]; }
    const double nr = sqrt(ta), nb = sqrt(tb);
    norms[0] = nr;
    norms[1] = nb;
    norms[2] = nb > 0.0 ? nr / nb : 0.0;
    S->ticket = 0u;
  }
}

// The CUDA context current on the calling thread (the driver's
// cuCtxGetCurrent, reached through the runtime so that no driver library
// is linked), or null when it cannot be asked.
using CtxGetCurrent = int (*)(void**);
void* current_context() {
  static CtxGetCurrent fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<CtxGetCurrent>(f);
  }();
  void* c = nullptr;
  if (!fn || fn(&c) != 0) return nullptr;
  return c;
}

void* g_na_ctx[kNaMaxDevices] = {nullptr};

// Device address of the scratch array on the current device, looked up
// once per device and context: after cudaDeviceReset (or any teardown of
// the device's context) the module is loaded again into the new context,
// where the array may sit at another address, so a change of the current
// context triggers a new lookup.
NaScratch* scratch_for_current_device(int* status) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNaMaxDevices) {
    *status = BP_ERR_NO_DEVICE;
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(g_na_mutex);
  void* ctx = current_context();
  if (!g_na_ptr[dev] || !ctx || ctx != g_na_ctx[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_na_scratch);
    if (e != cudaSuccess || !p) {
      std::fprintf(stderr, "bp_residual_noalloc: cudaGetSymbolAddress failed: %s\n",
                   cudaGetErrorString(e));
      *status = BP_ERR_CUDA;
      return nullptr;
    }
    g_na_ptr[dev] = static_cast<NaScratch*>(p);
    g_na_ctx[dev] = current_context();  // current now that the lookup made the runtime initialise it
  }
  *status = BP_OK;
  return g_na_ptr[dev];
}

}  // namespace

extern "C" int bp_residual_noalloc(int nx, int ny, int nz, int periodic,
                                   const int* active_vertex, const double* Auu,
                                   const double* Auv, const double* Avu, const double* Avv,
                                   const double* xu, const double* xv, const double* bu,
                                   const double* bv, double* resid_u, double* resid_v,
                                   double* norms, void* stream) {
  if (nx < 6 || ny < 6 || nz < 1) return BP_ERR_ARGS;
  if (!active_vertex || !Auu || !Auv || !Avu || !Avv || !xu || !xv || !bu || !bv || !resid_u ||
      !resid_v || !norms)
    return BP_ERR_ARGS;
  const long rows = (long)nz * (nx - 1) * (ny - 1);
  if (rows > kNaMaxRows) {
    std::fprintf(stderr,
                 "bp_residual_noalloc: %ld rows exceed the fixed scratch limit of %ld "
                 "(nz*(nx-1)*(ny-1)); use bp_matvec for larger systems\n",
                 rows, kNaMaxRows);
    return BP_ERR_ARGS;
  }
  int st = BP_OK;
  NaScratch* S = scratch_for_current_device(&st);
  if (!S) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(&S->ticket, 0, sizeof(unsigned), s) != cudaSuccess) return BP_ERR_CUDA;
  const unsigned blocks = (unsigned)((rows + kNaBlock - 1) / kNaBlock);
  k_resid_ref_layout<<<blocks, kNaBlock, 0, s>>>(nx, ny, nz, periodic, active_vertex, Auu, Auv,
                                                  Avu, Avv, xu, xv, bu, bv, resid_u, resid_v,
                                                  norms, S);
  return cudaGetLastError() == cudaSuccess ? BP_OK : BP_ERR_CUDA;
}
