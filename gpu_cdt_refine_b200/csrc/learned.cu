// Training and inference kernels of the learned Steiner placement network
// (no counterpart in the reference), and their C ABI.
//
// One warp carries 32 rows through the network: the forward pass of
// learned.cuh, then the backward pass with the same warp GEMM (bf16 operands
// on the tensor cores, fp32 accumulation).  Weight gradients of a warp go to
// its own slice of a partial-gradient buffer (no atomics, so the sum is
// deterministic); a second kernel sums the slices and a third applies Adam to
// the fp32 master parameters and refreshes their bf16 copies.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <random>
#include <vector>

#include "../../include/gqm_refine.h"
#include "learned.cuh"

namespace gqm {
namespace {

constexpr int kWarpsPerBlock = 2;

struct TrainSmem {
  uint16_t x[32 * kFeat];
  float h[32 * kHid];
  uint16_t a1[32 * kHid];
  uint16_t a2[32 * kHid];
  uint16_t dz[32 * kHid];
};

// The warp's 32 rows are positions base .. base+31 of a sequence of `end`
// rows; position p is row idx[off + p] (or off + p without idx).  Positions
// past the end are padding: zero features, no loss, no gradient.
__device__ __forceinline__ void load_rows(const float *X, const int *idx, long long off, long long base, long long end,
                                          uint16_t *x, int &row) {
  const int lane = (int)(threadIdx.x & 31u);
  const long long p = base + lane;
  row = p < end ? (idx ? idx[off + p] : (int)(off + p)) : -1;
  for (int j = 0; j < kFeat; ++j) x[lane * kFeat + j] = f2bf(row >= 0 ? X[(long long)row * kFeat + j] : 0.0f);
}

// inference as the placement step runs it (weights staged per block,
// activations in registers), kInferWarpsMax warps per block
__global__ void k_mlp_infer(MlpDev P, const float *X, long long n, float *out) {
  __shared__ MlpInferTiles sm;
  mlp_stage(P, sm.w);
  __syncthreads();
  const int warp = (int)(threadIdx.x >> 5), lane = (int)(threadIdx.x & 31u);
  uint16_t *x = sm.x[warp];
  const long long nw = (n + 31) / 32;
  for (long long gw = (long long)blockIdx.x * kInferWarpsMax + warp; gw < nw;
       gw += (long long)gridDim.x * kInferWarpsMax) {
    const long long row = gw * 32 + lane;
    float f[kFeat];
    if (row < n) {
      const float4 *xr = reinterpret_cast<const float4 *>(X + row * kFeat);
      for (int j = 0; j < kFeat / 4; ++j) {
        const float4 v = xr[j];
        f[4 * j] = v.x;
        f[4 * j + 1] = v.y;
        f[4 * j + 2] = v.z;
        f[4 * j + 3] = v.w;
      }
    } else {
      for (int j = 0; j < kFeat; ++j) f[j] = 0.0f;
    }
    mlp_put_row(x, lane, f);
    __syncwarp();
    const float y = mlp_forward_regs(sm.w, x);
    __syncwarp();
    if (row < n) out[row] = y;
  }
}
static int infer_blocks(long long n) {
  const long long nw = (n + 31) / 32;
  return (int)std::max<long long>(1, std::min<long long>((nw + kInferWarpsMax - 1) / kInferWarpsMax, 148 * 8));
}

// Forward and backward of rows [row0, row0 + nrows) (through idx when not
// null) with the loss  sum (y - t)^2 / denom.  Warp w writes its weight
// gradients to part[w][.] and its loss to lossp[w].
__global__ void k_mlp_fwd_bwd(MlpDev P, const float *X, const float *T, const int *idx, long long row0, long long nrows,
                              float denom, float *part, float *lossp) {
  __shared__ TrainSmem sm[kWarpsPerBlock];
  const int warp = (int)(threadIdx.x >> 5), lane = (int)(threadIdx.x & 31u);
  const int gw = (int)blockIdx.x * kWarpsPerBlock + warp;
  if ((long long)gw * 32 >= nrows) return;
  TrainSmem &s = sm[warp];
  float *g = part + (size_t)gw * kParamCount;
  int row;
  load_rows(X, idx, row0, (long long)gw * 32, nrows, s.x, row);
  const float y = mlp_forward_warp(P, s.x, s.h, s.a1, s.a2);
  const float err = row >= 0 ? y - T[row] : 0.0f;
  float l = err * err;
  for (int o = 16; o; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
  if (lane == 0) lossp[gw] = l / denom;
  const float dy = 2.0f * err / denom;
  // output layer
  for (int jj = 0; jj < kHid / 32; ++jj) {
    const int j = jj * 32 + lane;
    float gw3 = 0.0f;
    for (int r = 0; r < 32; ++r) {
      const float dyr = __shfl_sync(0xffffffffu, dy, r);
      gw3 += dyr * bf2f(s.a2[r * kHid + j]);
    }
    g[kOffW3 + j] = gw3;
  }
  float db3 = dy;
  for (int o = 16; o; o >>= 1) db3 += __shfl_xor_sync(0xffffffffu, db3, o);
  if (lane == 0) g[kOffB3] = db3;
  // dz2 = dy w3 [a2 > 0]  (bf16)
  for (int j = 0; j < kHid; ++j) {
    const float v = s.a2[lane * kHid + j] != 0 ? dy * bf2f(P.w3[j]) : 0.0f;
    s.dz[lane * kHid + j] = f2bf(v);
  }
  __syncwarp();
  // gW2[j][i] = sum_r dz2[r][j] a1[r][i]
  warp_gemm(kHid, kHid, 32, s.dz, 1, kHid, s.a1, kHid, 1, g + kOffW2, kHid, 1, false);
  __syncwarp();
  for (int jj = 0; jj < kHid / 32; ++jj) {
    const int j = jj * 32 + lane;
    float acc = 0.0f;
    for (int r = 0; r < 32; ++r) acc += bf2f(s.dz[r * kHid + j]);
    g[kOffB2 + j] = acc;
  }
  // dh1[r][i] = sum_j dz2[r][j] W2[j][i]
  warp_gemm(32, kHid, kHid, s.dz, kHid, 1, P.w2, kHid, 1, s.h, kHid, 1, false);
  __syncwarp();
  for (int i = 0; i < kHid; ++i) {
    const float v = s.a1[lane * kHid + i] != 0 ? s.h[lane * kHid + i] : 0.0f;
    s.dz[lane * kHid + i] = f2bf(v);
  }
  __syncwarp();
  // gW1[j][i] = sum_r dz1[r][j] x[r][i]
  warp_gemm(kHid, kFeat, 32, s.dz, 1, kHid, s.x, kFeat, 1, g + kOffW1, kFeat, 1, false);
  __syncwarp();
  for (int jj = 0; jj < kHid / 32; ++jj) {
    const int j = jj * 32 + lane;
    float acc = 0.0f;
    for (int r = 0; r < 32; ++r) acc += bf2f(s.dz[r * kHid + j]);
    g[kOffB1 + j] = acc;
  }
}

// grad[p] = sum over warps of part[w][p]; loss = sum of lossp
__global__ void k_mlp_reduce(const float *part, const float *lossp, int nw, float *grad, float *loss) {
  for (int p = (int)(blockIdx.x * blockDim.x + threadIdx.x); p < kParamCount; p += (int)(gridDim.x * blockDim.x)) {
    float acc = 0.0f;
    for (int w = 0; w < nw; ++w) acc += part[(size_t)w * kParamCount + p];
    grad[p] = acc;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    float acc = 0.0f;
    for (int w = 0; w < nw; ++w) acc += lossp[w];
    *loss = acc;
  }
}

// Adam on the fp32 master parameters; refreshes the bf16 weight copies.
__global__ void k_mlp_adam(float *params, float *m, float *v, const float *grad, float lr, float b1, float b2,
                           float eps, float c1, float c2, uint16_t *w1, uint16_t *w2, uint16_t *w3, float *bias) {
  for (int p = (int)(blockIdx.x * blockDim.x + threadIdx.x); p < kParamCount; p += (int)(gridDim.x * blockDim.x)) {
    const float gp = grad[p];
    const float mp = b1 * m[p] + (1.0f - b1) * gp, vp = b2 * v[p] + (1.0f - b2) * gp * gp;
    m[p] = mp;
    v[p] = vp;
    const float x = params[p] - lr * (mp / c1) / (sqrtf(vp / c2) + eps);
    params[p] = x;
    if (p < kOffB1)
      w1[p - kOffW1] = f2bf(x);
    else if (p < kOffW2)
      bias[p - kOffB1] = x;
    else if (p < kOffB2)
      w2[p - kOffW2] = f2bf(x);
    else if (p < kOffW3)
      bias[kHid + p - kOffB2] = x;
    else if (p < kOffB3)
      w3[p - kOffW3] = f2bf(x);
    else
      bias[2 * kHid] = x;
  }
}

// Device copy of a network: bf16 weights and fp32 biases (b1, b2, b3).
struct MlpBuf {
  uint16_t *w = nullptr;  // w1 | w2 | w3
  float *b = nullptr;     // b1 | b2 | b3
  MlpDev dev() const { return mlp_dev(w, b); }
  int upload(const float *params, cudaStream_t st) {
    if (!w && (cudaMalloc((void **)&w, sizeof(uint16_t) * kMlpW) != cudaSuccess ||
               cudaMalloc((void **)&b, sizeof(float) * kMlpB) != cudaSuccess))
      return GQM_ERR_MEMORY;
    std::vector<uint16_t> hw(kMlpW);
    std::vector<float> hb(kMlpB);
    mlp_pack(params, hw.data(), hb.data());
    if (cudaMemcpyAsync(w, hw.data(), sizeof(uint16_t) * hw.size(), cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(b, hb.data(), sizeof(float) * hb.size(), cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      return GQM_ERR_CUDA;
    return GQM_OK;
  }
  void release() {
    if (w) cudaFree(w);
    if (b) cudaFree(b);
    w = nullptr;
    b = nullptr;
  }
};

template <class T>
int dmalloc(T **p, size_t n) {
  return cudaMalloc((void **)p, sizeof(T) * (n ? n : 1)) == cudaSuccess ? GQM_OK : GQM_ERR_MEMORY;
}

// forward + backward + reduction over rows [row0, row0+nrows) of (X, T, idx)
int grad_pass(const MlpBuf &B, const float *dX, const float *dT, const int *didx, long long row0, long long nrows,
              float denom, float *dpart, float *dlossp, float *dgrad, float *dloss, cudaStream_t st) {
  const int nw = (int)((nrows + 31) / 32);
  const int blocks = (nw + kWarpsPerBlock - 1) / kWarpsPerBlock;
  k_mlp_fwd_bwd<<<blocks, 32 * kWarpsPerBlock, 0, st>>>(B.dev(), dX, dT, didx, row0, nrows, denom, dpart, dlossp);
  k_mlp_reduce<<<(kParamCount + 255) / 256, 256, 0, st>>>(dpart, dlossp, nw, dgrad, dloss);
  return cudaGetLastError() == cudaSuccess ? GQM_OK : GQM_ERR_CUDA;
}

}  // namespace
}  // namespace gqm

extern "C" {

int gqm_mlp_infer(int device, const float *params, const float *features, long long n, float *out) {
  using namespace gqm;
  if (!params || n < 0 || (n > 0 && (!features || !out))) return GQM_ERR_ARGUMENT;
  if (n == 0) return GQM_OK;
  if (cudaSetDevice(device) != cudaSuccess) return GQM_ERR_NO_DEVICE;
  cudaStream_t st;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return GQM_ERR_CUDA;
  MlpBuf B;
  float *dX = nullptr, *dY = nullptr;
  int rc = B.upload(params, st);
  if (!rc) rc = dmalloc(&dX, (size_t)n * kFeat);
  if (!rc) rc = dmalloc(&dY, (size_t)n);
  if (!rc) {
    cudaMemcpyAsync(dX, features, sizeof(float) * kFeat * n, cudaMemcpyHostToDevice, st);
    k_mlp_infer<<<infer_blocks(n), 32 * kInferWarpsMax, 0, st>>>(B.dev(), dX, n, dY);
    cudaMemcpyAsync(out, dY, sizeof(float) * n, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess || cudaGetLastError() != cudaSuccess) rc = GQM_ERR_CUDA;
  }
  if (dX) cudaFree(dX);
  if (dY) cudaFree(dY);
  B.release();
  cudaStreamDestroy(st);
  return rc;
}

int gqm_mlp_time(int device, const float *params, long long n, int iters, float *ms) {
  using namespace gqm;
  if (!params || !ms || n <= 0 || n > (1LL << 28) || iters <= 0) return GQM_ERR_ARGUMENT;
  if (cudaSetDevice(device) != cudaSuccess) return GQM_ERR_NO_DEVICE;
  cudaStream_t st;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return GQM_ERR_CUDA;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  MlpBuf B;
  float *dX = nullptr, *dY = nullptr;
  int rc = B.upload(params, st);
  if (!rc) rc = dmalloc(&dX, (size_t)n * kFeat);
  if (!rc) rc = dmalloc(&dY, (size_t)n);
  if (!rc && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)) rc = GQM_ERR_CUDA;
  if (!rc) {
    cudaMemsetAsync(dX, 0, sizeof(float) * kFeat * n, st);
    const int blocks = infer_blocks(n);
    k_mlp_infer<<<blocks, 32 * kInferWarpsMax, 0, st>>>(B.dev(), dX, n, dY);
    cudaEventRecord(e0, st);
    for (int i = 0; i < iters; ++i) k_mlp_infer<<<blocks, 32 * kInferWarpsMax, 0, st>>>(B.dev(), dX, n, dY);
    cudaEventRecord(e1, st);
    float t = 0.0f;
    if (cudaStreamSynchronize(st) != cudaSuccess || cudaGetLastError() != cudaSuccess ||
        cudaEventElapsedTime(&t, e0, e1) != cudaSuccess)
      rc = GQM_ERR_CUDA;
    else
      *ms = t / (float)iters;
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (dX) cudaFree(dX);
  if (dY) cudaFree(dY);
  B.release();
  cudaStreamDestroy(st);
  return rc;
}

int gqm_mlp_grad(int device, const float *params, const float *features, const float *targets, long long n,
                 float *loss, float *grad) {
  using namespace gqm;
  if (!params || !features || !targets || !loss || !grad || n <= 0 || n > (1LL << 24)) return GQM_ERR_ARGUMENT;
  if (cudaSetDevice(device) != cudaSuccess) return GQM_ERR_NO_DEVICE;
  cudaStream_t st;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return GQM_ERR_CUDA;
  MlpBuf B;
  float *dX = nullptr, *dT = nullptr, *dpart = nullptr, *dlp = nullptr, *dg = nullptr, *dl = nullptr;
  const int nw = (int)((n + 31) / 32);
  int rc = B.upload(params, st);
  if (!rc) rc = dmalloc(&dX, (size_t)n * kFeat) | dmalloc(&dT, (size_t)n) | dmalloc(&dpart, (size_t)nw * kParamCount) |
                dmalloc(&dlp, (size_t)nw) | dmalloc(&dg, (size_t)kParamCount) | dmalloc(&dl, 1);
  if (!rc) {
    cudaMemcpyAsync(dX, features, sizeof(float) * kFeat * n, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(dT, targets, sizeof(float) * n, cudaMemcpyHostToDevice, st);
    rc = grad_pass(B, dX, dT, nullptr, 0, n, (float)n, dpart, dlp, dg, dl, st);
    cudaMemcpyAsync(grad, dg, sizeof(float) * kParamCount, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(loss, dl, sizeof(float), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) rc = GQM_ERR_CUDA;
  }
  for (float *p : {dX, dT, dpart, dlp, dg, dl})
    if (p) cudaFree(p);
  B.release();
  cudaStreamDestroy(st);
  return rc;
}

int gqm_mlp_train(int device, float *params, const float *features, const float *targets, long long n, int epochs,
                  int batch, float lr, unsigned seed, float *loss) {
  using namespace gqm;
  if (!params || !features || !targets || n <= 0 || epochs < 0 || batch <= 0 || batch % 64 != 0 || !(lr > 0.0f))
    return GQM_ERR_ARGUMENT;
  if (cudaSetDevice(device) != cudaSuccess) return GQM_ERR_NO_DEVICE;
  cudaStream_t st;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return GQM_ERR_CUDA;
  MlpBuf B;
  float *dX = nullptr, *dT = nullptr, *dpart = nullptr, *dlp = nullptr, *dg = nullptr, *dl = nullptr;
  float *dp = nullptr, *dm = nullptr, *dv = nullptr;
  int *didx = nullptr;
  const int nw = batch / 32;
  int rc = B.upload(params, st);
  if (!rc)
    rc = dmalloc(&dX, (size_t)n * kFeat) | dmalloc(&dT, (size_t)n) | dmalloc(&dpart, (size_t)nw * kParamCount) |
         dmalloc(&dlp, (size_t)nw) | dmalloc(&dg, (size_t)kParamCount) | dmalloc(&dl, 1) |
         dmalloc(&dp, (size_t)kParamCount) | dmalloc(&dm, (size_t)kParamCount) | dmalloc(&dv, (size_t)kParamCount) |
         dmalloc(&didx, (size_t)n);
  float last = 0.0f;
  if (!rc) {
    cudaMemcpyAsync(dX, features, sizeof(float) * kFeat * n, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(dT, targets, sizeof(float) * n, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(dp, params, sizeof(float) * kParamCount, cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(dm, 0, sizeof(float) * kParamCount, st);
    cudaMemsetAsync(dv, 0, sizeof(float) * kParamCount, st);
    std::vector<int> perm(n);
    std::iota(perm.begin(), perm.end(), 0);
    std::mt19937 rng(seed);
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    long long step = 0;
    std::vector<float> lsum;
    for (int e = 0; e < epochs && !rc; ++e) {
      std::shuffle(perm.begin(), perm.end(), rng);
      cudaMemcpyAsync(didx, perm.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st);
      cudaStreamSynchronize(st);
      double esum = 0.0;
      long long nb = 0;
      for (long long r0 = 0; r0 < n && !rc; r0 += batch) {
        const long long rows = std::min<long long>(batch, n - r0);
        rc = grad_pass(B, dX, dT, didx, r0, rows, (float)rows, dpart, dlp, dg, dl, st);
        ++step;
        const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
        k_mlp_adam<<<(kParamCount + 255) / 256, 256, 0, st>>>(dp, dm, dv, dg, lr, b1, b2, eps, c1, c2, B.w,
                                                              B.w + kHid * kFeat, B.w + kHid * kFeat + kHid * kHid,
                                                              B.b);
        float hl = 0.0f;
        cudaMemcpyAsync(&hl, dl, sizeof(float), cudaMemcpyDeviceToHost, st);
        if (cudaStreamSynchronize(st) != cudaSuccess) rc = GQM_ERR_CUDA;
        esum += hl;
        ++nb;
      }
      last = nb ? (float)(esum / nb) : 0.0f;
    }
    if (!rc) {
      cudaMemcpyAsync(params, dp, sizeof(float) * kParamCount, cudaMemcpyDeviceToHost, st);
      if (cudaStreamSynchronize(st) != cudaSuccess) rc = GQM_ERR_CUDA;
    }
  }
  if (loss) *loss = last;
  for (float *p : {dX, dT, dpart, dlp, dg, dl, dp, dm, dv})
    if (p) cudaFree(p);
  if (didx) cudaFree(didx);
  B.release();
  cudaStreamDestroy(st);
  return rc;
}

}  // extern "C"
