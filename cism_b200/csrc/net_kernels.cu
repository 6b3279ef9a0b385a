// net_kernels.cu -- BF16 kernels of the learned initial guess: a 2-D
// U-Net over the vertex grid, trained and run on the device.
//
// Activations are NHWC ([pixel][channel]) in BF16; every contraction is a
// tensor-core GEMM on tcgen05 (k_gemm_tc: BF16 operands from shared memory,
// FP32 accumulator in tensor memory; the mma.sync kernel k_gemm_tn remains
// for comparison) over K-contiguous operands:
//   forward  Y[P][Cout]  = col(X)[P][K] . W[Cout][K]^T            (K = 9 Cin)
//   dgrad    dcol[P][K]  = dY[P][Cout] . WT[K][Cout]^T, then col2im
//   wgrad    dW[Cout][K] = dYT[Cout][P] . colT[K][P]^T
// with k = tap * Cin + c, tap = (dy + 1) * 3 + (dx + 1).  Borders are
// periodic (the doubly periodic domains) or zero.  Reductions (bias
// gradients, the loss) run in a fixed order, so a training run is
// deterministic.  Every entry point is extern "C" with plain device
// pointers and the CUDA stream to launch on.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <algorithm>
#include <cstdlib>
#include <map>
#include <mutex>
#include <cstring>

namespace {

typedef __nv_bfloat16 bf16;

// ---------------------------------------------------------------------
// GEMM: C[m][n] = sum_k A[m][k] B[n][k] (+ bias[n]) (+ C[m][n] if accum).
// Tiles 64 x 64 x 32, 4 warps of 32 x 32, cp.async double buffering.
// K, lda, ldb multiples of 8 (16-byte rows of the 8-element chunks).
// ---------------------------------------------------------------------
constexpr int BM = 64, BN = 64, BK = 32, PAD = 8;

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int n = valid ? 16 : 0;  // src-size 0: the 16 bytes are zero-filled
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(s), "l"(gmem), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

__device__ __forceinline__ void mma_bf16(float (&c)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__global__ void __launch_bounds__(128) k_gemm_tn(const bf16* __restrict__ A, const bf16* __restrict__ B,
                                                 float* __restrict__ C, const float* __restrict__ bias,
                                                 int M, int N, int K, int lda, int ldb, int ldc,
                                                 int accum) {
  __shared__ __align__(16) bf16 As[2][BM][BK + PAD];
  __shared__ __align__(16) bf16 Bs[2][BN][BK + PAD];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t4 = lane & 3;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  float acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.f;

  auto load = [&](int buf, int k0) {
#pragma unroll
    for (int c = 0; c < 2; ++c) {  // 64 rows x 4 chunks = 256 chunks per operand
      const int id = tid + c * 128;
      const int r = id >> 2, ch = (id & 3) * 8;
      const int k = k0 + ch;
      const bool va = (m0 + r) < M && k < K;
      const bool vb = (n0 + r) < N && k < K;
      cp_async16(&As[buf][r][ch], va ? (const void*)(A + (size_t)(m0 + r) * lda + k) : (const void*)A, va);
      cp_async16(&Bs[buf][r][ch], vb ? (const void*)(B + (size_t)(n0 + r) * ldb + k) : (const void*)B, vb);
    }
  };

  const int nk = (K + BK - 1) / BK;
  load(0, 0);
  cp_async_commit();
  for (int kt = 0; kt < nk; ++kt) {
    const int buf = kt & 1;
    if (kt + 1 < nk) {
      load(buf ^ 1, (kt + 1) * BK);
      cp_async_commit();
      cp_async_wait1();
    } else {
      cp_async_wait0();
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; kk += 16) {
      uint32_t af[2][4], bfr[4][2];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int r = wm + i * 16 + g;
        af[i][0] = *reinterpret_cast<const uint32_t*>(&As[buf][r][kk + 2 * t4]);
        af[i][1] = *reinterpret_cast<const uint32_t*>(&As[buf][r + 8][kk + 2 * t4]);
        af[i][2] = *reinterpret_cast<const uint32_t*>(&As[buf][r][kk + 2 * t4 + 8]);
        af[i][3] = *reinterpret_cast<const uint32_t*>(&As[buf][r + 8][kk + 2 * t4 + 8]);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int nn = wn + j * 8 + g;
        bfr[j][0] = *reinterpret_cast<const uint32_t*>(&Bs[buf][nn][kk + 2 * t4]);
        bfr[j][1] = *reinterpret_cast<const uint32_t*>(&Bs[buf][nn][kk + 2 * t4 + 8]);
      }
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) mma_bf16(acc[i][j], af[i], bfr[j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int m = m0 + wm + i * 16 + g + (q >> 1) * 8;
        const int n = n0 + wn + j * 8 + 2 * t4 + (q & 1);
        if (m < M && n < N) {
          float x = acc[i][j][q];
          if (bias) x += bias[n];
          float* dst = C + (size_t)m * ldc + n;
          *dst = accum ? *dst + x : x;
        }
      }
}

// ---------------------------------------------------------------------
// im2col / col2im over [B][H][W][C] with 3 x 3 taps; periodic != 0 wraps.
// ---------------------------------------------------------------------
__device__ __forceinline__ bool tap_pixel(int b, int y, int x, int dy, int dx, int H, int W, int periodic,
                                          long long* p) {
  int yy = y + dy, xx = x + dx;
  if (periodic) {
    yy = (yy + H) % H;
    xx = (xx + W) % W;
  } else if (yy < 0 || yy >= H || xx < 0 || xx >= W) {
    return false;
  }
  *p = ((long long)b * H + yy) * W + xx;
  return true;
}

__global__ void k_im2col(const bf16* __restrict__ X, bf16* __restrict__ col, int B, int H, int W, int C,
                         int Kp, int periodic) {
  const long long total = (long long)B * H * W * Kp;
  for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < total;
       id += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(id % Kp);
    const long long p = id / Kp;
    bf16 val = __float2bfloat16(0.f);
    if (k < 9 * C) {
      const int tap = k / C, c = k - tap * C;
      const int x = (int)(p % W), y = (int)((p / W) % H), b = (int)(p / ((long long)W * H));
      long long q;
      if (tap_pixel(b, y, x, tap / 3 - 1, tap % 3 - 1, H, W, periodic, &q)) val = X[q * C + c];
    }
    col[id] = val;
  }
}

// dX[p][c] = sum over taps of dcol[q][tap * C + c], q the pixel whose tap
// lands on p (gather in tap order).
__global__ void k_col2im(const float* __restrict__ dcol, float* __restrict__ dX, int B, int H, int W, int C,
                         int Kp, int periodic) {
  const long long total = (long long)B * H * W * C;
  for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < total;
       id += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(id % C);
    const long long p = id / C;
    const int x = (int)(p % W), y = (int)((p / W) % H), b = (int)(p / ((long long)W * H));
    float s = 0.f;
    for (int tap = 0; tap < 9; ++tap) {
      long long q;
      if (tap_pixel(b, y, x, -(tap / 3 - 1), -(tap % 3 - 1), H, W, periodic, &q))
        s += dcol[q * Kp + tap * C + c];
    }
    dX[id] = s;
  }
}

// [R][Cc] -> [Cc][R] (BF16), 32 x 32 tiles through shared memory.
__global__ void k_transpose(const bf16* __restrict__ in, bf16* __restrict__ out, int R, int Cc) {
  __shared__ bf16 tile[32][33];
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int r = r0 + i, c = c0 + threadIdx.x;
    if (r < R && c < Cc) tile[i][threadIdx.x] = in[(size_t)r * Cc + c];
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int c = c0 + i, r = r0 + threadIdx.x;
    if (r < R && c < Cc) out[(size_t)c * R + r] = tile[threadIdx.x][i];
  }
}

// ---------------------------------------------------------------------
// pointwise
// ---------------------------------------------------------------------
__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
  const float cdf = 0.5f * (1.f + erff(x * 0.70710678118654752f));
  const float pdf = 0.39894228040143268f * expf(-0.5f * x * x);
  return cdf + x * pdf;
}

#define GRID_LOOP(id, total) \
  for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < (total); id += (long long)gridDim.x * blockDim.x)

// Y = act(Z) in BF16 into a channel slice [p][c0 .. c0 + C) of rows of ldy.
__global__ void k_act(const float* __restrict__ Z, bf16* __restrict__ Y, long long P, int C, int ldy, int c0,
                      int act) {
  GRID_LOOP(id, P * C) {
    const long long p = id / C;
    const int c = (int)(id % C);
    const float z = Z[id];
    Y[p * ldy + c0 + c] = __float2bfloat16(act ? gelu(z) : z);
  }
}

// dZ = dY * act'(Z), dY read from a channel slice of rows of ldd (FP32).
__global__ void k_act_grad(const float* __restrict__ Z, const float* __restrict__ dY, float* __restrict__ dZ,
                           long long P, int C, int ldd, int c0, int act) {
  GRID_LOOP(id, P * C) {
    const long long p = id / C;
    const int c = (int)(id % C);
    const float d = dY[p * ldd + c0 + c];
    dZ[id] = act ? d * gelu_grad(Z[id]) : d;
  }
}

__global__ void k_f32_to_bf16(const float* __restrict__ x, bf16* __restrict__ y, long long n) {
  GRID_LOOP(id, n) y[id] = __float2bfloat16(x[id]);
}

// Column sums db[c] = sum_p dZ[p][c] (fixed order: one thread per column
// strides the rows, then a fixed-shape tree within the block).
__global__ void k_colsum(const float* __restrict__ dZ, float* __restrict__ db, long long P, int C) {
  __shared__ float sm[256];
  const int c = blockIdx.x;
  float s = 0.f;
  for (long long p = threadIdx.x; p < P; p += blockDim.x) s += dZ[p * C + c];
  sm[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sm[threadIdx.x] += sm[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) db[c] = sm[0];
}

// 2 x 2 average pooling, [B][H][W][C] -> [B][H/2][W/2][C] (BF16).
__global__ void k_pool(const bf16* __restrict__ X, bf16* __restrict__ Y, int B, int H, int W, int C) {
  const int h = H / 2, w = W / 2;
  GRID_LOOP(id, (long long)B * h * w * C) {
    const int c = (int)(id % C);
    const long long p = id / C;
    const int x = (int)(p % w), y = (int)((p / w) % h), b = (int)(p / ((long long)w * h));
    const long long q = ((long long)b * H + 2 * y) * W + 2 * x;
    const float s = __bfloat162float(X[q * C + c]) + __bfloat162float(X[(q + 1) * C + c]) +
                    __bfloat162float(X[(q + W) * C + c]) + __bfloat162float(X[(q + W + 1) * C + c]);
    Y[id] = __float2bfloat16(0.25f * s);
  }
}

// gradient of the pooling: dX[fine] += dY[coarse] / 4 (FP32, channel slice
// of the coarse rows)
__global__ void k_pool_grad(const float* __restrict__ dY, float* __restrict__ dX, int B, int H, int W, int C,
                            int ldy, int c0) {
  GRID_LOOP(id, (long long)B * H * W * C) {
    const int c = (int)(id % C);
    const long long p = id / C;
    const int x = (int)(p % W), y = (int)((p / W) % H), b = (int)(p / ((long long)W * H));
    const long long q = ((long long)b * (H / 2) + y / 2) * (W / 2) + x / 2;
    dX[id] += 0.25f * dY[q * ldy + c0 + c];
  }
}

// nearest 2x upsampling of [B][h][w][C] into a channel slice of the fine
// rows (ldy)
__global__ void k_up(const bf16* __restrict__ X, bf16* __restrict__ Y, int B, int h, int w, int C, int ldy,
                     int c0) {
  const int H = 2 * h, W = 2 * w;
  GRID_LOOP(id, (long long)B * H * W * C) {
    const int c = (int)(id % C);
    const long long p = id / C;
    const int x = (int)(p % W), y = (int)((p / W) % H), b = (int)(p / ((long long)W * H));
    const long long q = ((long long)b * h + y / 2) * w + x / 2;
    Y[p * ldy + c0 + c] = X[q * C + c];
  }
}

// gradient of the upsampling: dX[coarse] = sum of its 4 fine pixels (fixed order)
__global__ void k_up_grad(const float* __restrict__ dY, float* __restrict__ dX, int B, int h, int w, int C,
                          int ldy, int c0) {
  const int W = 2 * w;
  GRID_LOOP(id, (long long)B * h * w * C) {
    const int c = (int)(id % C);
    const long long p = id / C;
    const int x = (int)(p % w), y = (int)((p / w) % h), b = (int)(p / ((long long)w * h));
    const long long q = ((long long)b * 2 * h + 2 * y) * W + 2 * x;
    dX[id] = dY[q * ldy + c0 + c] + dY[(q + 1) * ldy + c0 + c] + dY[(q + W) * ldy + c0 + c] +
             dY[(q + W + 1) * ldy + c0 + c];
  }
}

// copy a BF16 [P][C] block into a channel slice of rows of ldy
__global__ void k_copy_slice(const bf16* __restrict__ X, bf16* __restrict__ Y, long long P, int C, int ldy,
                             int c0) {
  GRID_LOOP(id, P * C) {
    const long long p = id / C;
    const int c = (int)(id % C);
    Y[p * ldy + c0 + c] = X[id];
  }
}

// dX += a channel slice of dY (FP32)
__global__ void k_add_slice(const float* __restrict__ dY, float* __restrict__ dX, long long P, int C, int ldy,
                            int c0) {
  GRID_LOOP(id, P * C) {
    const long long p = id / C;
    const int c = (int)(id % C);
    dX[id] += dY[p * ldy + c0 + c];
  }
}

// Masked mean squared error over [P][C] (mask per pixel): per-block
// partial sums in a fixed order; gradient 2 (y - t) mask / count.
__global__ void k_mse(const float* __restrict__ Y, const float* __restrict__ T, const float* __restrict__ mask,
                      float* __restrict__ dY, float* __restrict__ partial, long long P, int C, float inv_count) {
  __shared__ float sm[256];
  float s = 0.f;
  for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < P * C;
       id += (long long)gridDim.x * blockDim.x) {
    const float m = mask[id / C];
    const float e = (Y[id] - T[id]) * m;
    dY[id] = 2.f * e * inv_count;
    s += e * e;
  }
  sm[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sm[threadIdx.x] += sm[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = sm[0] * inv_count;
}

// Adam on FP32 master weights; the BF16 GEMM copy W[Cout][Kp] (k < K real,
// the padding stays zero) is refreshed in the same pass.
__global__ void k_adam(float* __restrict__ w, const float* __restrict__ grad, float* __restrict__ m1,
                       float* __restrict__ m2, bf16* __restrict__ wb, long long n, int K, int Kp, float lr,
                       float b1, float b2, float eps, float c1, float c2) {
  GRID_LOOP(id, n) {
    const float gr = grad[id];
    const float a = b1 * m1[id] + (1.f - b1) * gr;
    const float b = b2 * m2[id] + (1.f - b2) * gr * gr;
    m1[id] = a;
    m2[id] = b;
    const float x = w[id] - lr * (a * c1) / (sqrtf(b * c2) + eps);
    w[id] = x;
    if (wb) {
      const long long r = id / K;
      const int k = (int)(id % K);
      wb[r * Kp + k] = __float2bfloat16(x);
    }
  }
}

// gradient of a padded BF16 GEMM weight [Cout][Kp] back to [Cout][K]
__global__ void k_unpad(const float* __restrict__ src, float* __restrict__ dst, long long rows, int K, int Kp) {
  GRID_LOOP(id, rows * K) {
    const long long r = id / K;
    const int k = (int)(id % K);
    dst[id] = src[r * Kp + k];
  }
}

inline unsigned grid_for(long long n) {
  long long g = (n + 255) / 256;
  if (g > 65535LL * 16) g = 65535LL * 16;
  return (unsigned)(g < 1 ? 1 : g);
}

// ---------------------------------------------------------------------
// The same GEMM on the 5th-generation tensor cores (tcgen05): one CTA of
// four warps per 128 x 64 tile of C, its FP32 accumulator in tensor memory
// (64 of the SM's 512 TMEM columns, lane = row), the operands staged in
// shared memory in the K-major no-swizzle core-matrix layout (8 rows x 16
// bytes per 128-byte core matrix) that the UMMA shared-memory descriptor
// describes, two stages deep: while the tensor core multiplies one 64-deep
// K slice the threads load the next.  One thread issues the four K = 16
// tcgen05.mma of a slice and commits them to the stage's mbarrier; the
// stage is refilled once that barrier completes.  The epilogue reads the
// accumulator with tcgen05.ld (warp w: rows 32w..32w+31) and adds the bias
// (and C) through shared memory, so that stores run along rows.  Every
// wait is bounded: past the limit the kernel raises g_tc_err, stops
// issuing, frees its tensor memory and returns.
// ---------------------------------------------------------------------
constexpr int TC_BM = 128, TC_BK = 64;
constexpr int TC_A_BYTES = TC_BM * TC_BK * 2;
// BN = 64, 32 for the products with at most 32 output columns, or 128
template <int BN>
constexpr int tc_stage_bytes() { return TC_A_BYTES + BN * TC_BK * 2; }  // 20, 24 or 32 KB

__device__ int g_tc_err = 0;  // a wait of k_gemm_tc ran out (read and cleared by bpnet_gemm_status)

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// UMMA shared-memory descriptor, K-major, no swizzle: start address, leading
// byte offset (between the two 16-byte K chunks of one K = 16 step), stride
// byte offset (between 8-row groups), version 1, base offset 0, layout 0.
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator (bits 4-5 = 1), A
// and B BF16 (bits 7-9, 10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4
// at bit 24.
template <int BN>
constexpr uint32_t tc_idesc() {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(TC_BM >> 4) << 24);
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (int i = 0; i < (1 << 24); ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  atomicExch(&g_tc_err, 1);
  return false;
}

// Split K: CTA z of the grid covers K slices [z * kchunk, min(K, (z + 1) *
// kchunk)) (kchunk a multiple of TC_BK) and writes its partial product to
// C + z * cstride; gridDim.z = 1 is the whole K with bias and accumulation.
template <int BN>
__global__ void __launch_bounds__(128) k_gemm_tc(const bf16* __restrict__ A, const bf16* __restrict__ B,
                                                 float* __restrict__ C, const float* __restrict__ bias,
                                                 int M, int N, int K, int lda, int ldb, int ldc,
                                                 int accum, int kchunk, long long cstride) {
  extern __shared__ __align__(1024) uint8_t tc_smem[];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ uint32_t tmem_slot;
  const int tid = threadIdx.x, warp = tid >> 5;
  constexpr int STAGE = tc_stage_bytes<BN>();
  const int m0 = blockIdx.y * TC_BM, n0 = blockIdx.x * BN;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"(BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar[0])));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar[1])));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;
  const int kbeg = blockIdx.z * kchunk, kend = min(K, kbeg + kchunk);
  C += (size_t)blockIdx.z * cstride;
  const int nk = (kend - kbeg + TC_BK - 1) / TC_BK;
  bool ok = true;
  for (int it = 0; it < nk; ++it) {
    const int st = it & 1;
    uint8_t* As = tc_smem + st * STAGE;
    uint8_t* Bs = As + TC_A_BYTES;
    if (it >= 2) ok = mbar_wait(smem_u32(&bar[st]), ((it - 2) >> 1) & 1);  // the stage's last slice is done
    if (!__syncthreads_and(ok)) {
      ok = false;
      break;
    }
    const int k0 = kbeg + it * TC_BK;
    for (int c = tid; c < TC_BM * 8; c += 128) {  // 128 rows x 8 chunks of 8 K elements
      const int r = c >> 3, kc = c & 7, gm = m0 + r, gk = k0 + kc * 8;
      uint4 val = make_uint4(0u, 0u, 0u, 0u);
      if (gm < M && gk < kend) val = __ldg(reinterpret_cast<const uint4*>(A + (size_t)gm * lda + gk));
      *reinterpret_cast<uint4*>(As + (kc * (TC_BM / 8) + (r >> 3)) * 128 + (r & 7) * 16) = val;
    }
    for (int c = tid; c < BN * 8; c += 128) {
      const int r = c >> 3, kc = c & 7, gn = n0 + r, gk = k0 + kc * 8;
      uint4 val = make_uint4(0u, 0u, 0u, 0u);
      if (gn < N && gk < kend) val = __ldg(reinterpret_cast<const uint4*>(B + (size_t)gn * ldb + gk));
      *reinterpret_cast<uint4*>(Bs + (kc * (BN / 8) + (r >> 3)) * 128 + (r & 7) * 16) = val;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // the tensor core reads through the async proxy
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
      for (int s = 0; s < TC_BK / 16; ++s) {
        if (k0 + 16 * s >= kend) break;
        const uint64_t ad = umma_desc(smem_u32(As) + 2 * s * (TC_BM / 8) * 128, (TC_BM / 8) * 128, 128);
        const uint64_t bd = umma_desc(smem_u32(Bs) + 2 * s * (BN / 8) * 128, (BN / 8) * 128, 128);
        const uint32_t acc = (it > 0 || s > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
            ::"r"(tmem), "l"(ad), "l"(bd), "r"(tc_idesc<BN>()), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(&bar[st]))
                   : "memory");
    }
  }
  // the last commit completes after every multiply of the tile (the host
  // never launches an empty K range)
  if (ok) ok = mbar_wait(smem_u32(&bar[(nk - 1) & 1]), ((nk - 1) >> 1) & 1);
  ok = __syncthreads_and(ok);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (ok) {
    // warp w holds rows 32w..32w+31 of the tile (one row per lane); each
    // 32 x 32 block goes through shared memory (the stages are free now)
    // so that a store instruction writes 32 consecutive columns of a row
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // after the tensor core's reads of the stages
    float* T = reinterpret_cast<float*>(tc_smem) + warp * (32 * 33);
    const int lane = tid & 31;
#pragma unroll
    for (int c0 = 0; c0 < BN; c0 += 32) {
      uint32_t v[32];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
          "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
            "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
            "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),
            "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
          : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int j = 0; j < 32; ++j) T[lane * 33 + j] = __uint_as_float(v[j]);
      __syncwarp();
      const int col = n0 + c0 + lane;
      if (col < N) {
        const float bc = bias ? bias[col] : 0.f;
        for (int r = 0; r < 32; ++r) {
          const int row = m0 + warp * 32 + r;
          if (row >= M) break;
          float* dst = C + (size_t)row * ldc + col;
          float x = T[r * 33 + lane] + bc;
          if (accum) x += *dst;
          *dst = x;
        }
      }
      __syncwarp();
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN));
}

// ---------------------------------------------------------------------
// The same product with its operands brought in by the Tensor Memory
// Accelerator: a four-stage ring of shared-memory slices, each filled by
// 16 cp.async.bulk.tensor boxes (one K chunk of 8 elements by 128 rows of
// A, or by BN rows of B: exactly one column of core matrices of the
// no-swizzle K-major layout, so the boxes land where the UMMA descriptors
// read) that complete on the stage's "full" mbarrier.  One thread issues
// the loads and the tcgen05.mma of every slice; a stage is refilled with
// the slice four ahead once the tensor core's commit for it has arrived on
// the stage's "done" mbarrier, so up to four slices of loads are in flight
// while the tensor core works.  Out-of-range rows and K columns read as
// zero (the tensor maps' bounds).  Epilogue as k_gemm_tc.  Every wait is
// bounded; on a timeout the issuing thread waits (bounded) for its copies
// and its last multiply in flight, raises g_tc_err, and the CTA frees its
// tensor memory and returns.  Loads only: no TMA store, no multicast.
// ---------------------------------------------------------------------
constexpr int TM_STAGES = 4;

template <int BN>
constexpr int tm_smem_bytes() { return TM_STAGES * tc_stage_bytes<BN>() + 1024; }  // + room to align the ring

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%1], %0;" ::"r"(bytes), "r"(bar) : "memory");
}

// A box of the 2-D tensor map at (x = K element, y = row) into shared
// memory; x is always a multiple of 8 (16 bytes).
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::
          "r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(x), "r"(y)
      : "memory");
}

template <int BN>
__global__ void __launch_bounds__(128) k_gemm_tma(const __grid_constant__ CUtensorMap tmA,
                                                  const __grid_constant__ CUtensorMap tmB, float* __restrict__ C,
                                                  const float* __restrict__ bias, int M, int N, int K, int ldc,
                                                  int accum, int kchunk, long long cstride) {
  extern __shared__ __align__(1024) uint8_t tc_smem[];
  __shared__ __align__(8) uint64_t full[TM_STAGES], done[TM_STAGES];
  __shared__ uint32_t tmem_slot;
  __shared__ int s_ok;
  constexpr int STAGE = tc_stage_bytes<BN>();
  const int tid = threadIdx.x, warp = tid >> 5;
  const int m0 = blockIdx.y * TC_BM, n0 = blockIdx.x * BN;
  const int kbeg = blockIdx.z * kchunk, kend = min(K, kbeg + kchunk);
  C += (size_t)blockIdx.z * cstride;
  const int nk = (kend - kbeg + TC_BK - 1) / TC_BK;
  // the ring starts on a 1024-byte boundary (the boxes land on 512-byte ones)
  const uint32_t ring = (smem_u32(tc_smem) + 1023u) & ~1023u;
  uint8_t* ring_ptr = tc_smem + (ring - smem_u32(tc_smem));
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"(BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int st = 0; st < TM_STAGES; ++st) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&full[st])));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&done[st])));
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_ok = 1;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;
  if (tid == 0) {
    auto issue = [&](int j) {  // slice j into stage j % TM_STAGES
      const int st = j % TM_STAGES;
      const uint32_t a = ring + st * STAGE, b = a + TC_A_BYTES, bar = smem_u32(&full[st]);
      mbar_expect_tx(bar, STAGE);
      const int k0 = kbeg + j * TC_BK;
#pragma unroll
      for (int kc = 0; kc < 8; ++kc) {
        tma_load_2d(a + kc * (TC_BM / 8) * 128, &tmA, k0 + kc * 8, m0, bar);
        tma_load_2d(b + kc * (BN / 8) * 128, &tmB, k0 + kc * 8, n0, bar);
      }
    };
    bool ok = true;
    int issued = 0, it = 0, last_mma = -1;
    for (; issued < nk && issued < TM_STAGES; ++issued) issue(issued);
    for (; it < nk; ++it) {
      const int st = it % TM_STAGES;
      if (!mbar_wait(smem_u32(&full[st]), (it / TM_STAGES) & 1)) {
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int k0 = kbeg + it * TC_BK;
      const uint32_t a = ring + st * STAGE, b = a + TC_A_BYTES;
#pragma unroll
      for (int s = 0; s < TC_BK / 16; ++s) {
        if (k0 + 16 * s >= kend) break;
        const uint64_t ad = umma_desc(a + 2 * s * (TC_BM / 8) * 128, (TC_BM / 8) * 128, 128);
        const uint64_t bd = umma_desc(b + 2 * s * (BN / 8) * 128, (BN / 8) * 128, 128);
        const uint32_t acc = (it > 0 || s > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem),
            "l"(ad), "l"(bd), "r"(tc_idesc<BN>()), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(&done[st]))
                   : "memory");
      last_mma = it;
      if (issued < nk) {  // the stage takes the slice TM_STAGES ahead once this multiply has read it
        if (!mbar_wait(smem_u32(&done[st]), (it / TM_STAGES) & 1)) {
          ok = false;
          ++it;
          break;
        }
        issue(issued);
        ++issued;
      }
    }
    if (ok && last_mma >= 0)  // the last commit completes after every multiply of the tile
      ok = mbar_wait(smem_u32(&done[last_mma % TM_STAGES]), (last_mma / TM_STAGES) & 1);
    if (!ok) {  // no copy and no multiply may still be in flight when the CTA exits
      for (int j = it; j < issued; ++j) mbar_wait(smem_u32(&full[j % TM_STAGES]), (j / TM_STAGES) & 1);
      if (last_mma >= 0) mbar_wait(smem_u32(&done[last_mma % TM_STAGES]), (last_mma / TM_STAGES) & 1);
      s_ok = 0;
    }
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (s_ok) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // after the copies and the tensor core's reads
    float* T = reinterpret_cast<float*>(ring_ptr) + warp * (32 * 33);
    const int lane = tid & 31;
#pragma unroll
    for (int c0 = 0; c0 < BN; c0 += 32) {
      uint32_t v[32];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
          "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
            "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
            "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),
            "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
          : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int j = 0; j < 32; ++j) T[lane * 33 + j] = __uint_as_float(v[j]);
      __syncwarp();
      const int col = n0 + c0 + lane;
      if (col < N) {
        const float bc = bias ? bias[col] : 0.f;
        for (int r = 0; r < 32; ++r) {
          const int row = m0 + warp * 32 + r;
          if (row >= M) break;
          float* dst = C + (size_t)row * ldc + col;
          float x = T[r * 33 + lane] + bc;
          if (accum) x += *dst;
          *dst = x;
        }
      }
      __syncwarp();
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN));
}

// The 2-D tensor map of a row-major BF16 operand [rows][ld] (K = the first
// K columns) with boxes of 8 K elements by box_rows rows; false where the
// driver has no encoder or refuses the operand (address or stride not
// 16-byte aligned).
bool tma_map(CUtensorMap* map, const void* ptr, int rows, int K, int ld, int box_rows) {
  static PFN_cuTensorMapEncodeTiled_v12000 enc = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  }();
  if (!enc || (reinterpret_cast<uintptr_t>(ptr) & 15) || ((size_t)ld * 2) % 16) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  const cuuint32_t box[2] = {8, (cuuint32_t)box_rows};
  const cuuint32_t es[2] = {1, 1};
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims, strides, box, es,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// C[r][c] = sum over z of part[z][r][c] in z order (+ bias) (+ C): the
// split-K partial products, summed deterministically.
__global__ void k_splitk_sum(const float* __restrict__ part, int S, long long cstride, float* __restrict__ C,
                             const float* __restrict__ bias, int M, int N, int ldc, int accum) {
  GRID_LOOP(id, (long long)M * N) {
    const long long r = id / N;
    const int c = (int)(id % N);
    float v = 0.f;
    for (int z = 0; z < S; ++z) v += part[z * cstride + id];
    if (bias) v += bias[c];
    float* dst = C + r * ldc + c;
    if (accum) v += *dst;
    *dst = v;
  }
}

// Grow-only scratch of the split-K partial products, one per device (the
// current one); a buffer is replaced only after the device has finished
// with it.
float* splitk_scratch(size_t n) {
  static std::mutex mu;
  static std::map<int, std::pair<float*, size_t>> bufs;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  std::lock_guard<std::mutex> lock(mu);
  auto& b = bufs[dev];
  if (n > b.second) {
    if (b.first) {
      cudaDeviceSynchronize();
      cudaFree(b.first);
    }
    b = {nullptr, 0};
    if (cudaMalloc(&b.first, n * sizeof(float)) != cudaSuccess) return nullptr;
    b.second = n;
  }
  return b.first;
}

// One tcgen05 product of tile width W: TMA-fed (maps given) or register-staged.
template <int W>
void launch_tile(bool tma, const CUtensorMap& ma, const CUtensorMap& mb, dim3 grid, cudaStream_t st,
                 const bf16* A, const bf16* B, float* out, const float* bout, int M, int N, int K, int lda, int ldb,
                 int ldo, int acc, int kchunk, long long cs) {
  if (tma)
    k_gemm_tma<W><<<grid, 128, tm_smem_bytes<W>(), st>>>(ma, mb, out, bout, M, N, K, ldo, acc, kchunk, cs);
  else
    k_gemm_tc<W><<<grid, 128, 2 * tc_stage_bytes<W>(), st>>>(A, B, out, bout, M, N, K, lda, ldb, ldo, acc, kchunk,
                                                             cs);
}

template <int W>
bool tile_smem_ok() {
  return cudaFuncSetAttribute(k_gemm_tc<W>, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * tc_stage_bytes<W>()) ==
             cudaSuccess &&
         cudaFuncSetAttribute(k_gemm_tma<W>, cudaFuncAttributeMaxDynamicSharedMemorySize, tm_smem_bytes<W>()) ==
             cudaSuccess;
}

}  // namespace

extern "C" {

// Returns 0, or 10 for arguments the kernels do not take.  A product
// with few output tiles and a long K (the weight gradients, K = pixels)
// is split along K over enough CTAs to fill the GPU, its partial products
// summed in order by k_splitk_sum.
// The product with an explicit kernel: mode 0 tcgen05 with TMA-fed operands
// (k_gemm_tma), 1 tcgen05 with register-staged operands (k_gemm_tc), 2 the
// mma.sync kernel.
int bpnet_gemm_tn_mode(int mode, const void* A, const void* B, float* C, const float* bias, int M, int N, int K,
                       int lda, int ldb, int ldc, int accum, void* stream) {
  if (M <= 0 || N <= 0 || K <= 0 || (K % 8) || (lda % 8) || (ldb % 8) || mode < 0 || mode > 2) return 10;
  static const bool smem_ok = tile_smem_ok<32>() && tile_smem_ok<64>() && tile_smem_ok<128>();
  if (!smem_ok) return 6;
  cudaStream_t st = (cudaStream_t)stream;
  if (mode == 2) {
    dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM);
    k_gemm_tn<<<grid, 128, 0, st>>>((const bf16*)A, (const bf16*)B, C, bias, M, N, K, lda, ldb, ldc, accum);
    return cudaGetLastError() == cudaSuccess ? 0 : 6;
  }
  // tile width: 32 for at most 32 columns (no MMA work on padding); 128
  // for widths that are not a multiple of 64 where it pads no more than 64
  // does (96: one tile instead of 64 + 32, A read once); else 64 (a
  // multiple of 64 keeps twice the CTAs: 128 x 128 tiles measured slower at
  // N = 128 and 1152)
  int bn = 64;
  if (N <= 32)
    bn = 32;
  else if (N % 64 != 0 && (N + 127) / 128 * 128 <= (N + 63) / 64 * 64)
    bn = 128;
  const int gx = (N + bn - 1) / bn, gy = (M + TC_BM - 1) / TC_BM, nslices = (K + TC_BK - 1) / TC_BK;
  int S = 1, kchunk = nslices * TC_BK;
  if (gx * gy < 296 && nslices >= 64) S = std::min((296 + gx * gy - 1) / (gx * gy), nslices / 16);
  float* out = C;
  const float* bout = bias;
  int ldo = ldc, acc = accum;
  long long cs = 0;
  if (S > 1) {  // partial products into the scratch, summed afterwards
    kchunk = (nslices + S - 1) / S * TC_BK;
    S = (K + kchunk - 1) / kchunk;  // no empty chunk
    cs = (long long)M * N;
    out = splitk_scratch((size_t)S * cs);
    if (!out) return 6;
    bout = nullptr;
    ldo = N;
    acc = 0;
  }
  const dim3 grid(gx, gy, S);
  CUtensorMap ma, mb;
  // a product of one K slice has no pipeline to fill: the register-staged
  // kernel starts sooner (measured faster at K <= 64, slower above)
  const bool tma =
      mode == 0 && nslices > 1 && tma_map(&ma, A, M, K, lda, TC_BM) && tma_map(&mb, B, N, K, ldb, bn);
  const bf16 *a16 = (const bf16*)A, *b16 = (const bf16*)B;
  if (bn == 32)
    launch_tile<32>(tma, ma, mb, grid, st, a16, b16, out, bout, M, N, K, lda, ldb, ldo, acc, kchunk, cs);
  else if (bn == 64)
    launch_tile<64>(tma, ma, mb, grid, st, a16, b16, out, bout, M, N, K, lda, ldb, ldo, acc, kchunk, cs);
  else
    launch_tile<128>(tma, ma, mb, grid, st, a16, b16, out, bout, M, N, K, lda, ldb, ldo, acc, kchunk, cs);
  if (S > 1) k_splitk_sum<<<grid_for(cs), 256, 0, st>>>(out, S, cs, C, bias, M, N, ldc, accum);
  return cudaGetLastError() == cudaSuccess ? 0 : 6;
}

// The product on the default kernel: tcgen05 with TMA-fed operands (with
// register-staged ones for a single K slice); BPNET_GEMM=tc selects the
// register-staged tcgen05 kernel throughout, BPNET_GEMM=mma the mma.sync one.
int bpnet_gemm_tn(const void* A, const void* B, float* C, const float* bias, int M, int N, int K, int lda,
                  int ldb, int ldc, int accum, void* stream) {
  static const int mode = [] {
    const char* e = std::getenv("BPNET_GEMM");
    if (e && std::strcmp(e, "mma") == 0) return 2;
    if (e && std::strcmp(e, "tc") == 0) return 1;
    return 0;
  }();
  return bpnet_gemm_tn_mode(mode, A, B, C, bias, M, N, K, lda, ldb, ldc, accum, stream);
}

// The mma.sync kernel (the comparison of the tcgen05 one).
int bpnet_gemm_tn_mma(const void* A, const void* B, float* C, const float* bias, int M, int N, int K, int lda,
                      int ldb, int ldc, int accum, void* stream) {
  if (M <= 0 || N <= 0 || K <= 0 || (K % 8) || (lda % 8) || (ldb % 8)) return 10;
  dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM);
  k_gemm_tn<<<grid, 128, 0, (cudaStream_t)stream>>>((const bf16*)A, (const bf16*)B, C, bias, M, N, K, lda,
                                                     ldb, ldc, accum);
  return cudaGetLastError() == cudaSuccess ? 0 : 6;
}

// 1 if a wait of the tcgen05 GEMM ran out since the last call (and clears
// it), 0 if not, 6 on a CUDA error.
int bpnet_gemm_status(void* stream) {
  int e = 0, z = 0;
  if (cudaMemcpyFromSymbolAsync(&e, g_tc_err, sizeof(int), 0, cudaMemcpyDeviceToHost, (cudaStream_t)stream) !=
          cudaSuccess ||
      cudaMemcpyToSymbolAsync(g_tc_err, &z, sizeof(int), 0, cudaMemcpyHostToDevice, (cudaStream_t)stream) !=
          cudaSuccess ||
      cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess)
    return 6;
  return e;
}

int bpnet_im2col(const void* X, void* col, int B, int H, int W, int C, int Kp, int periodic, void* stream) {
  const long long n = (long long)B * H * W * Kp;
  k_im2col<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>((const bf16*)X, (bf16*)col, B, H, W, C, Kp, periodic);
  return cudaGetLastError() == cudaSuccess ? 0 : 6;
}

int bpnet_col2im(const float* dcol, float* dX, int B, int H, int W, int C, int Kp, int periodic, void* stream) {
  const long long n = (long long)B * H * W * C;
  k_col2im<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(dcol, dX, B, H, W, C, Kp, periodic);
  return cudaGetLastError() == cudaSuccess ? 0 : 6;
}

int bpnet_transpose(const void* in, void* out, int R, int Cc, void* stream) {
  dim3 grid((Cc + 31) / 32, (R + 31) / 32), block(32, 8);
  k_transpose<<<grid, block, 0, (cudaStream_t)stream>>>((const bf16*)in, (bf16*)out, R, Cc);
  return cudaGetLastError() == cudaSuccess ? 0 : 6;
}

int bpnet_act(const float* Z, void* Y, long long P, int C, int ldy, int c0, int act, void* stream) {
  k_act<<<grid_for(P * C), 256, 0, (cudaStream_t)stream>>>(Z, (bf16*)Y, P, C, ldy, c0, act);
  return cudaGetLastError() == cudaSuccess ? 0 : 6;
}

int bpnet_act_grad(const float* Z, const float* dY, float* dZ, long long P, int C, int ldd, int c0, int act,
                   void* stream) {
  k_act_grad<<<grid_for(P * C), 256, 0, (cudaStream_t)stream>>>(Z, dY, dZ, P, C, ldd, c0, act);
  return cudaGetLastError() == cudaSuccess ? 0 : 6;
}

int bpnet_to_bf16(const float* x, void* y, long long n, void* stream) {
  k_f32_to_bf16<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(x, (bf16*)y, n);
  return cudaGetLastError() == cudaSuccess ? 0 : 6;
}

int bpnet_colsum(const float* dZ, float* db, long long P, int C, void* stream) {
  k_colsum<<<C, 256, 0, (cudaStream_t)stream>>>(dZ, db, P, C);
  return cudaGetLastError() == cudaSuccess ? 0 : 6;
}

int bpnet_pool(const void* X, void* Y, int B, int H, int W, int C, void* stream) {
  if ((H % 2) || (W % 2)) return 10;
  const long long n = (long long)B * (H / 2) * (W / 2) * C;
  k_pool<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>((const bf16*)X, (bf16*)Y, B, H, W, C);
  return cudaGetLastError() == cudaSuccess ? 0 : 6;
}

int bpnet_pool_grad(const float* dY, float* dX, int B, int H, int W, int C, int ldy, int c0, void* stream) {
  const long long n = (long long)B * H * W * C;
  k_pool_grad<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(dY, dX, B, H, W, C, ldy, c0);
  return cudaGetLastError() == cudaSuccess ? 0 : 6;
}

int bpnet_up(const void* X, void* Y, int B, int h, int w, int C, int ldy, int c0, void* stream) {
  const long long n = (long long)B * 4 * h * w * C;
  k_up<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>((const bf16*)X, (bf16*)Y, B, h, w, C, ldy, c0);
  return cudaGetLastError() == cudaSuccess ? 0 : 6;
}

int bpnet_up_grad(const float* dY, float* dX, int B, int h, int w, int C, int ldy, int c0, void* stream) {
  const long long n = (long long)B * h * w * C;
  k_up_grad<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(dY, dX, B, h, w, C, ldy, c0);
  return cudaGetLastError() == cudaSuccess ? 0 : 6;
}

int bpnet_copy_slice(const void* X, void* Y, long long P, int C, int ldy, int c0, void* stream) {
  k_copy_slice<<<grid_for(P * C), 256, 0, (cudaStream_t)stream>>>((const bf16*)X, (bf16*)Y, P, C, ldy, c0);
  return cudaGetLastError() == cudaSuccess ? 0 : 6;
}

int bpnet_add_slice(const float* dY, float* dX, long long P, int C, int ldy, int c0, void* stream) {
  k_add_slice<<<grid_for(P * C), 256, 0, (cudaStream_t)stream>>>(dY, dX, P, C, ldy, c0);
  return cudaGetLastError() == cudaSuccess ? 0 : 6;
}

// partial must hold 256 floats; the loss is the sum of them (host side).
int bpnet_mse(const float* Y, const float* T, const float* mask, float* dY, float* partial, long long P, int C,
              float inv_count, void* stream) {
  k_mse<<<256, 256, 0, (cudaStream_t)stream>>>(Y, T, mask, dY, partial, P, C, inv_count);
  return cudaGetLastError() == cudaSuccess ? 0 : 6;
}

int bpnet_adam(float* w, const float* grad, float* m1, float* m2, void* wb, long long n, int K, int Kp,
               float lr, float b1, float b2, float eps, float c1, float c2, void* stream) {
  k_adam<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(w, grad, m1, m2, (bf16*)wb, n, K, Kp, lr, b1, b2, eps,
                                                        c1, c2);
  return cudaGetLastError() == cudaSuccess ? 0 : 6;
}

int bpnet_unpad(const float* src, float* dst, long long rows, int K, int Kp, void* stream) {
  k_unpad<<<grid_for(rows * K), 256, 0, (cudaStream_t)stream>>>(src, dst, rows, K, Kp);
  return cudaGetLastError() == cudaSuccess ? 0 : 6;
}

}  // extern "C"
