// bp_guess.cu -- the learned initial guess behind the C ABI.
//
// The reference starts the Picard loop from the caller's velocity (the last
// time step's, glissade.F90:1919-1987).  With bp_inputs.guess_mode =
// BP_GUESS_LEARNED the library replaces that start by a U-Net's estimate,
// computed on the device from the problem's own device arrays and written
// straight into the problem's initial velocity; the unchanged Picard/PCG
// solve then converges to the same tolerance from it.
//
// Network (net.py holds the training side): a 2-D U-Net on the owned
// vertex grid padded to multiples of 8, four levels of two 3 x 3
// convolutions with GELU, 2 x 2 average pooling, nearest upsampling with
// skip concatenation, a 1 x 1 head; BF16 weights and activations, FP32
// accumulation.  Inputs at each active column: thickness (km), the driving
// stress (the column's gravity load per horizontal area, 1e5 Pa) in x and
// y, log10 of beta (>= 1), and +1 / -1 for grounded / floating ice (beta >
// 0 or not); zero at inactive vertices.  Outputs: (u, v) on each level,
// scaled by the training set's RMS speed.  Every layer runs in this
// library's kernels (net_kernels.cu); the weights come from the flat
// binary file net.UNet.save_bin writes.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "bp_guess.h"

extern "C" {
int bpnet_gemm_tn(const void* A, const void* B, float* C, const float* bias, int M, int N, int K, int lda,
                  int ldb, int ldc, int accum, void* stream);
int bpnet_im2col(const void* X, void* col, int B, int H, int W, int C, int Kp, int periodic, void* stream);
int bpnet_act(const float* Z, void* Y, long long P, int C, int ldy, int c0, int act, void* stream);
int bpnet_pool(const void* X, void* Y, int B, int H, int W, int C, void* stream);
int bpnet_up(const void* X, void* Y, int B, int h, int w, int C, int ldy, int c0, void* stream);
int bpnet_copy_slice(const void* X, void* Y, long long P, int C, int ldy, int c0, void* stream);
}

namespace bp {

namespace {

using bf16 = __nv_bfloat16;

struct GConv {
  int cin, cout, k3, act, K, Kp;
  bf16* wb = nullptr;  // [cout][Kp], zero past K
  float* b = nullptr;  // [cout]
};

int ceil8(int x) { return (x + 7) / 8 * 8; }

}  // namespace

struct GuessNet {
  int nin = 0, nout = 0;
  std::vector<int> ch;
  std::vector<GConv> convs;
  float shift[8] = {0}, scale[8] = {0}, out_scale = 1.f;
  std::map<std::string, std::pair<void*, size_t>> ws;  // device workspace, grow-only

  void* get(const char* name, size_t bytes) {
    bytes = std::max<size_t>((bytes + 255) / 256 * 256, 256);
    auto it = ws.find(name);
    if (it != ws.end() && it->second.second >= bytes) return it->second.first;
    if (it != ws.end()) {
      cudaDeviceSynchronize();
      cudaFree(it->second.first);
      ws.erase(it);
    }
    void* p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
    ws[name] = {p, bytes};
    return p;
  }
  ~GuessNet() {
    for (auto& c : convs) {
      cudaFree(c.wb);
      cudaFree(c.b);
    }
    for (auto& kv : ws) cudaFree(kv.second.first);
  }
};

GuessNet* guess_net_load(const char* path, std::string* err) {
  FILE* f = std::fopen(path, "rb");
  if (!f) {
    *err = std::string("cannot open ") + path;
    return nullptr;
  }
  auto rd = [&](void* dst, size_t bytes) { return std::fread(dst, 1, bytes, f) == bytes; };
  char magic[8];
  int hdr[4];
  GuessNet* N = new GuessNet();
  bool ok = rd(magic, 8) && std::memcmp(magic, "BPUNET1", 8) == 0 && rd(hdr, sizeof(hdr)) && hdr[0] == 1 &&
            (hdr[1] == 5 || hdr[1] == 6) && hdr[2] > 0 && hdr[2] % 8 == 0 && hdr[3] >= 1 && hdr[3] <= 8;
  int nconv = 0;
  if (ok) {
    N->nin = hdr[1];
    N->nout = hdr[2];
    N->ch.resize(hdr[3]);
    ok = rd(N->ch.data(), sizeof(int) * hdr[3]) && rd(&nconv, sizeof(int)) && nconv == 4 * hdr[3] - 1 &&
         rd(N->shift, sizeof(float) * N->nin) && rd(N->scale, sizeof(float) * N->nin) && rd(&N->out_scale, 4);
  }
  for (int i = 0; ok && i < nconv; ++i) {
    int d[5];
    ok = rd(d, sizeof(d)) && d[1] > 0 && d[1] % 8 == 0 && d[4] == (d[2] ? 9 * d[0] : d[0]);
    if (!ok) break;
    GConv c;
    c.cin = d[0]; c.cout = d[1]; c.k3 = d[2]; c.act = d[3]; c.K = d[4]; c.Kp = ceil8(c.K);
    std::vector<float> w((size_t)c.cout * c.K), b(c.cout);
    ok = rd(w.data(), sizeof(float) * w.size()) && rd(b.data(), sizeof(float) * b.size());
    if (!ok) break;
    std::vector<bf16> wb((size_t)c.cout * c.Kp, __float2bfloat16_rn(0.f));
    for (int o = 0; o < c.cout; ++o)
      for (int k = 0; k < c.K; ++k) wb[(size_t)o * c.Kp + k] = __float2bfloat16_rn(w[(size_t)o * c.K + k]);
    ok = cudaMalloc(&c.wb, sizeof(bf16) * wb.size()) == cudaSuccess &&
         cudaMalloc(&c.b, sizeof(float) * b.size()) == cudaSuccess &&
         cudaMemcpy(c.wb, wb.data(), sizeof(bf16) * wb.size(), cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(c.b, b.data(), sizeof(float) * b.size(), cudaMemcpyHostToDevice) == cudaSuccess;
    N->convs.push_back(c);
  }
  std::fclose(f);
  ok = ok && !N->convs.empty() && N->convs[0].cin == N->nin;
  if (!ok) {
    *err = std::string("malformed U-Net weights file ") + path;
    delete N;
    return nullptr;
  }
  return N;
}

void guess_net_free(GuessNet* N) { delete N; }

namespace {

// Features of one instance's active columns, normalised and rounded to
// BF16, into grid b of x [B][H][W][nin] (the grid is zeroed beforehand).
// The arithmetic follows net.input_features / net.normalized_input.
__global__ void k_guess_features(DevView v, int col_begin, int col_end, int ilo, int jlo, int H, int W, int b,
                                 double area, GuessNorm nrm, bf16* x) {
  const int col = col_begin + blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= col_end) return;
  double su = 0.0, sv = 0.0;
  for (int k = 0; k < v.nz; ++k) {
    const double2 l = v.load[node_of(v, col, k)];
    su = su + l.x;
    sv = sv + l.y;
  }
  const double beta = v.col_beta[col];
  double f[6] = {v.col_h[col] / 1000.0, su * area, sv * area, log10(fmax(beta, 1.0)), beta > 0.0 ? 1.0 : -1.0, 0.0};
  if (nrm.nin > 5) {  // mean flwafact over the layers of the column's active cells (SW, SE, NW, NE of the vertex)
    double sf = 0.0, cnt = 0.0;
    for (int q = 0; q < 4; ++q) {
      const int c = v.col_cells[q * v.ncols + col];
      if (c < 0) continue;
      for (int k = 0; k < v.nz - 1; ++k) {
        sf = sf + v.flwafact[(size_t)c * (v.nz - 1) + k];
        cnt = cnt + 1.0;
      }
    }
    f[5] = cnt > 0.0 ? log10(sf / cnt) : 0.0;
  }
  const int gi = v.col_ij[col] - ilo, gj = v.col_ij[v.ncols + col] - jlo;
  bf16* dst = x + (((size_t)b * H + gj) * W + gi) * nrm.nin;
  for (int c = 0; c < nrm.nin; ++c)
    dst[c] = __float2bfloat16_rn(__double2float_rn((f[c] - (double)nrm.shift[c]) * (double)nrm.scale[c]));
}

// The network's output of grid b at each column of the instance, times the
// output scale (in FP32, as the training side does), into x0 (node order).
__global__ void k_guess_scatter(DevView v, int col_begin, int col_end, int ilo, int jlo, int H, int W, int b,
                                int nout, float out_scale, const float* out, double2* x0) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int nz = v.nz;
  if (t >= (long)(col_end - col_begin) * nz) return;
  const int col = col_begin + (int)(t / nz), k = (int)(t % nz);
  const int gi = v.col_ij[col] - ilo, gj = v.col_ij[v.ncols + col] - jlo;
  const float* o = out + (((size_t)b * H + gj) * W + gi) * nout;
  const float u = o[2 * k] * out_scale, w = o[2 * k + 1] * out_scale;
  x0[node_of(v, col, k)] = make_double2((double)u, (double)w);
}

#define NK(call)                 \
  do {                           \
    if ((call) != 0) return 6;   \
  } while (0)

// One convolution: x [P][cin] BF16 -> y [P][cout] BF16 (and z, FP32 pre-activation).
int conv_fwd(GuessNet* N, const GConv& c, const bf16* x, bf16* y, int B, int H, int W, int periodic,
             cudaStream_t s, int* nl) {
  *nl += (c.k3 ? 1 : 0) + 1 + (y ? 1 : 0);
  const long long P = (long long)B * H * W;
  const bf16* col = x;
  if (c.k3) {
    bf16* cb = (bf16*)N->get("col", sizeof(bf16) * (size_t)P * c.Kp);
    if (!cb) return 6;
    NK(bpnet_im2col(x, cb, B, H, W, c.cin, c.Kp, periodic, s));
    col = cb;
  }
  float* z = (float*)N->get(y ? "z" : "head", sizeof(float) * (size_t)P * c.cout);
  if (!z) return 6;
  NK(bpnet_gemm_tn(col, c.wb, z, c.b, (int)P, c.cout, c.Kp, c.Kp, c.Kp, c.cout, 0, s));
  if (y) NK(bpnet_act(z, y, P, c.cout, c.cout, 0, c.act, s));
  return 0;
}

// The U-Net forward of net.UNet.forward: x [B][H][W][5] BF16 -> FP32
// [B][H][W][nout] in the workspace "head".
int unet_forward(GuessNet* N, const bf16* x, int B, int H, int W, int periodic, cudaStream_t s, float** out,
                 int* nlaunch) {
  const int nl = (int)N->ch.size();
  std::vector<bf16*> skip(nl);
  const bf16* cur = x;
  int ci = 0;
  const size_t P0 = (size_t)B * H * W;
  size_t act = 0;  // the largest activation: level lv holds P0 / 4^lv points of ch[lv] channels
  for (int lv = 0; lv < nl; ++lv) act = std::max(act, (P0 >> (2 * lv)) * (size_t)N->ch[lv]);
  bf16* bufA = (bf16*)N->get("act_a", sizeof(bf16) * act);
  bf16* bufB = (bf16*)N->get("act_b", sizeof(bf16) * act);
  if (!bufA || !bufB) return 6;
  for (int lv = 0; lv < nl; ++lv) {
    const int h = H >> lv, w = W >> lv;
    if (lv > 0) {
      NK(bpnet_pool(cur, bufA, B, H >> (lv - 1), W >> (lv - 1), N->ch[lv - 1], s));
      ++*nlaunch;
      cur = bufA;
    }
    NK(conv_fwd(N, N->convs[ci], cur, bufB, B, h, w, periodic, s, nlaunch));
    ++ci;
    char nm[16];
    std::snprintf(nm, sizeof(nm), "skip%d", lv);
    skip[lv] = (bf16*)N->get(nm, sizeof(bf16) * (size_t)B * h * w * N->ch[lv]);
    if (!skip[lv]) return 6;
    NK(conv_fwd(N, N->convs[ci], bufB, skip[lv], B, h, w, periodic, s, nlaunch));
    ++ci;
    cur = skip[lv];
  }
  for (int lv = nl - 2; lv >= 0; --lv) {
    const int h = H >> lv, w = W >> lv;
    const int cu = N->ch[lv + 1], cs = N->ch[lv];
    const long long P = (long long)B * h * w;
    bf16* cat = (bf16*)N->get("cat", sizeof(bf16) * (size_t)P * (cu + cs));
    if (!cat) return 6;
    NK(bpnet_up(cur, cat, B, h / 2, w / 2, cu, cu + cs, 0, s));
    NK(bpnet_copy_slice(skip[lv], cat, P, cs, cu + cs, cu, s));
    *nlaunch += 2;
    NK(conv_fwd(N, N->convs[ci], cat, bufA, B, h, w, periodic, s, nlaunch));
    ++ci;
    NK(conv_fwd(N, N->convs[ci], bufA, bufB, B, h, w, periodic, s, nlaunch));
    ++ci;
    cur = bufB;
  }
  NK(conv_fwd(N, N->convs[ci], cur, nullptr, B, H, W, periodic, s, nlaunch));
  *out = (float*)N->get("head", 0);
  return 0;
}

}  // namespace

int guess_net_run(GuessNet* N, const HostPlan& p, const DevView& v, const std::vector<int>& which, double2* x0,
                  cudaStream_t s, int* launches) {
  int nlaunch = 0;
  if (p.solve2d || p.nz * 2 > N->nout) return BP_ERR_ARGS;
  GuessNorm nrm;
  nrm.nin = N->nin;
  for (int c = 0; c < N->nin; ++c) {
    nrm.shift[c] = N->shift[c];
    nrm.scale[c] = N->scale[c];
  }
  // instances of one padded grid shape and border type run as one batch
  std::map<std::tuple<int, int, int>, std::vector<int>> groups;
  for (int b : which) {
    const OwnedRange R = owned_range(p.nx[b], p.ny[b], p.periodic[b]);
    groups[{ceil8(R.jhi - R.jlo + 1), ceil8(R.ihi - R.ilo + 1), p.periodic[b]}].push_back(b);
  }
  for (auto& g : groups) {
    const int H = std::get<0>(g.first), W = std::get<1>(g.first), per = std::get<2>(g.first);
    const int B = (int)g.second.size();
    bf16* x = (bf16*)N->get("input", sizeof(bf16) * (size_t)B * H * W * N->nin);
    if (!x) return BP_ERR_CUDA;
    if (cudaMemsetAsync(x, 0, sizeof(bf16) * (size_t)B * H * W * N->nin, s) != cudaSuccess) return BP_ERR_CUDA;
    for (int bi = 0; bi < B; ++bi) {
      const int b = g.second[bi];
      const InstParams& ip = p.inst[b];
      const OwnedRange R = owned_range(p.nx[b], p.ny[b], p.periodic[b]);
      const int nc = ip.col_end - ip.col_begin;
      const double area = 1.0e9 / (ip.dx * ip.dy) * 1.0e-5;
      if (nc > 0) {
        k_guess_features<<<(nc + 255) / 256, 256, 0, s>>>(v, ip.col_begin, ip.col_end, R.ilo, R.jlo, H, W, bi,
                                                          area, nrm, x);
        ++nlaunch;
      }
    }
    float* out = nullptr;
    if (unet_forward(N, x, B, H, W, per, s, &out, &nlaunch) != 0) return BP_ERR_CUDA;
    for (int bi = 0; bi < B; ++bi) {
      const int b = g.second[bi];
      const InstParams& ip = p.inst[b];
      const OwnedRange R = owned_range(p.nx[b], p.ny[b], p.periodic[b]);
      const long n = (long)(ip.col_end - ip.col_begin) * p.nz;
      if (n > 0) {
        k_guess_scatter<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(v, ip.col_begin, ip.col_end, R.ilo, R.jlo, H,
                                                                     W, bi, N->nout, N->out_scale, out, x0);
        ++nlaunch;
      }
    }
  }
  if (launches) *launches += nlaunch;
  return cudaGetLastError() == cudaSuccess ? BP_OK : BP_ERR_CUDA;
}

}  // namespace bp
