// Learned Steiner placement (no counterpart in the reference; it attaches
// where the reference computes a bad triangle's Steiner point,
// computeCircumcenter, GPU_Refine/refine.cu:3780-3868).
//
// The off-center of the reference lies on the bisector of the triangle's
// shortest edge, at offConstant edge lengths from the edge's midpoint, and is
// used when it is nearer than the circumcenter.  In that case the learned rule
// places the point at
//     s = s_off + t (s_cc - s_off),   t = MLP(features) clamped to [0, 1],
// between the off-center (t = 0) and the circumcenter (t = 1), s counted in
// edge lengths along the bisector.  The plain off-center is kept whenever the
// clamp binds (t <= 0 or t >= 1) or the proposed point encroaches a
// subsegment of the triangle or of its neighbours.
//
// The network: 32 fp32 features -> 64 -> 64 -> 1, ReLU, weights in bf16, fp32
// accumulation on the tensor cores (mma.sync m16n8k16, bf16 x bf16 -> fp32),
// biases in fp32.  The same warp-level GEMM serves inference and training.
#pragma once
#include <cstdint>

#include "gqm_device.cuh"

namespace gqm {

constexpr int kFeat = 32, kHid = 64;
// fp32 parameter vector: W1[64][32], b1[64], W2[64][64], b2[64], w3[64], b3
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kHid * kFeat, kOffW2 = kOffB1 + kHid, kOffB2 = kOffW2 + kHid * kHid,
              kOffW3 = kOffB2 + kHid, kOffB3 = kOffW3 + kHid, kParamCount = kOffB3 + 1;

// bf16 as raw bits: round to nearest even from fp32 (finite inputs)
__host__ __device__ inline uint16_t f2bf(float f) {
  uint32_t u;
  memcpy(&u, &f, 4);
  u += 0x7FFFu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}
__host__ __device__ inline float bf2f(uint16_t h) {
  uint32_t u = (uint32_t)h << 16;
  float f;
  memcpy(&f, &u, 4);
  return f;
}

// Network in device memory: bf16 weights (row-major, out x in) and fp32 biases.
struct MlpDev {
  const uint16_t *w1, *w2, *w3;
  const float *b1, *b2, *b3;
};
// Packed device form: weights w1 | w2 | w3 (bf16), biases b1 | b2 | b3 (fp32).
constexpr int kMlpW = kHid * kFeat + kHid * kHid + kHid, kMlpB = 2 * kHid + 1;
__host__ __device__ inline MlpDev mlp_dev(const uint16_t *w, const float *b) {
  return MlpDev{w, w + kHid * kFeat, w + kHid * kFeat + kHid * kHid, b, b + kHid, b + 2 * kHid};
}
inline void mlp_pack(const float *params, uint16_t *w, float *b) {
  for (int i = 0; i < kHid * kFeat; ++i) w[i] = f2bf(params[kOffW1 + i]);
  for (int i = 0; i < kHid * kHid; ++i) w[kHid * kFeat + i] = f2bf(params[kOffW2 + i]);
  for (int i = 0; i < kHid; ++i) w[kHid * kFeat + kHid * kHid + i] = f2bf(params[kOffW3 + i]);
  for (int i = 0; i < kHid; ++i) b[i] = params[kOffB1 + i];
  for (int i = 0; i < kHid; ++i) b[kHid + i] = params[kOffB2 + i];
  b[2 * kHid] = params[kOffB3];
}

// ---------------------------------------------------------------------------
// Warp GEMM on shared-memory operands: C[i][j] (+)= sum_k A(i,k) B(k,j) with
// A(i,k) = a[i*ai + k*ak], B(k,j) = b[k*bk + j*bj] (bf16 bits), M % 16 == 0,
// N % 8 == 0, K % 16 == 0; C(i,j) = c[i*ci + j*cj] in fp32.  Called by all 32
// lanes of a warp.  Fragment layout of mma.m16n8k16 (PTX ISA): lane = 4 g + q;
// A regs (g, 2q..2q+1), (g+8, 2q..), (g, 2q+8..), (g+8, 2q+8..); B regs
// (2q..2q+1, g), (2q+8.., g); C (g, 2q..2q+1), (g+8, 2q..2q+1).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t pack2(uint16_t lo, uint16_t hi) { return (uint32_t)lo | ((uint32_t)hi << 16); }
__device__ inline void warp_gemm(int M, int N, int K, const uint16_t *a, int ai, int ak, const uint16_t *b, int bk,
                                 int bj, float *c, int ci, int cj, bool accumulate) {
#ifdef GQM_HOST_EMU
  for (int i = 0; i < M; ++i)
    for (int j = 0; j < N; ++j) {
      float s = accumulate ? c[i * ci + j * cj] : 0.0f;
      for (int k = 0; k < K; ++k) s += bf2f(a[i * ai + k * ak]) * bf2f(b[k * bk + j * bj]);
      c[i * ci + j * cj] = s;
    }
#else
  const int lane = (int)(threadIdx.x & 31u), g = lane >> 2, q = lane & 3;
  for (int i0 = 0; i0 < M; i0 += 16)
    for (int j0 = 0; j0 < N; j0 += 8) {
      float d[4];
      d[0] = accumulate ? c[(i0 + g) * ci + (j0 + 2 * q) * cj] : 0.0f;
      d[1] = accumulate ? c[(i0 + g) * ci + (j0 + 2 * q + 1) * cj] : 0.0f;
      d[2] = accumulate ? c[(i0 + g + 8) * ci + (j0 + 2 * q) * cj] : 0.0f;
      d[3] = accumulate ? c[(i0 + g + 8) * ci + (j0 + 2 * q + 1) * cj] : 0.0f;
      for (int k0 = 0; k0 < K; k0 += 16) {
        const uint16_t *A = a + i0 * ai + k0 * ak;
        const uint16_t *B = b + k0 * bk + j0 * bj;
        uint32_t ra[4], rb[2];
        ra[0] = pack2(A[g * ai + (2 * q) * ak], A[g * ai + (2 * q + 1) * ak]);
        ra[1] = pack2(A[(g + 8) * ai + (2 * q) * ak], A[(g + 8) * ai + (2 * q + 1) * ak]);
        ra[2] = pack2(A[g * ai + (2 * q + 8) * ak], A[g * ai + (2 * q + 9) * ak]);
        ra[3] = pack2(A[(g + 8) * ai + (2 * q + 8) * ak], A[(g + 8) * ai + (2 * q + 9) * ak]);
        rb[0] = pack2(B[(2 * q) * bk + g * bj], B[(2 * q + 1) * bk + g * bj]);
        rb[1] = pack2(B[(2 * q + 8) * bk + g * bj], B[(2 * q + 9) * bk + g * bj]);
        asm volatile(
            "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
            "{%0,%1,%2,%3};\n"
            : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
            : "r"(ra[0]), "r"(ra[1]), "r"(ra[2]), "r"(ra[3]), "r"(rb[0]), "r"(rb[1]));
      }
      __syncwarp();
      c[(i0 + g) * ci + (j0 + 2 * q) * cj] = d[0];
      c[(i0 + g) * ci + (j0 + 2 * q + 1) * cj] = d[1];
      c[(i0 + g + 8) * ci + (j0 + 2 * q) * cj] = d[2];
      c[(i0 + g + 8) * ci + (j0 + 2 * q + 1) * cj] = d[3];
      __syncwarp();
    }
#endif
}

// Forward pass of 32 rows (row r = lane r) held in x (bf16, 32 x 32) in shared
// memory; h (fp32, 32 x 64) and a1 (bf16, 32 x 64) are shared scratch, a2
// (bf16, 32 x 64) keeps the second layer's activations when not null.
// Returns this lane's output.  Weights are read from global memory (bf16).
__device__ inline float mlp_forward_warp(const MlpDev &P, const uint16_t *x, float *h, uint16_t *a1, uint16_t *a2) {
  const int lane = (int)(threadIdx.x & 31u);
  __syncwarp();
  // layer 1: h = x W1^T
  warp_gemm(32, kHid, kFeat, x, kFeat, 1, P.w1, 1, kFeat, h, kHid, 1, false);
  __syncwarp();
  for (int j = 0; j < kHid; ++j) {
    const float v = h[lane * kHid + j] + P.b1[j];
    a1[lane * kHid + j] = f2bf(v > 0.0f ? v : 0.0f);
  }
  __syncwarp();
  // layer 2: h = a1 W2^T
  warp_gemm(32, kHid, kHid, a1, kHid, 1, P.w2, 1, kHid, h, kHid, 1, false);
  __syncwarp();
  float y = P.b3[0];
  for (int j = 0; j < kHid; ++j) {
    const float v = h[lane * kHid + j] + P.b2[j];
    const uint16_t hb = f2bf(v > 0.0f ? v : 0.0f);
    if (a2) a2[lane * kHid + j] = hb;
    y += bf2f(hb) * bf2f(P.w3[j]);
  }
  __syncwarp();
  return y;
}
// The same network for one row with scalar arithmetic (the CPU emulation of
// the tests runs kernels one thread at a time, without warps).
__host__ __device__ inline float mlp_forward_row(const MlpDev &P, const float *f) {
  float a1[kHid], y = P.b3[0];
  for (int j = 0; j < kHid; ++j) {
    float z = 0.0f;
    for (int k = 0; k < kFeat; ++k) z += bf2f(f2bf(f[k])) * bf2f(P.w1[j * kFeat + k]);
    z += P.b1[j];
    a1[j] = bf2f(f2bf(z > 0.0f ? z : 0.0f));
  }
  for (int j = 0; j < kHid; ++j) {
    float z = 0.0f;
    for (int k = 0; k < kHid; ++k) z += a1[k] * bf2f(P.w2[j * kHid + k]);
    z += P.b2[j];
    y += bf2f(f2bf(z > 0.0f ? z : 0.0f)) * bf2f(P.w3[j]);
  }
  return y;
}
struct MlpInferSmem {
  uint16_t x[32 * kFeat];
  float h[32 * kHid];
  uint16_t a1[32 * kHid];
};

// ---------------------------------------------------------------------------
// Inference with the weights staged in shared memory once per block and the
// activations kept in registers: the accumulator fragments of two adjacent
// 8-column tiles of one layer are, after bias, ReLU and bf16 rounding, the A
// fragment of a 16-column step of the next layer (mma.m16n8k16 layouts, as in
// warp_gemm above).  Rows of the weight and input tiles are padded by 8 bf16
// so that the fragment loads of a warp hit 32 distinct banks.  Layers 1 and 2
// round exactly as mlp_forward_warp; layer 3 sums a lane's 16 columns and then
// the four lanes of a quad, so its fp32 rounding order differs from the
// sequential sum there.
// ---------------------------------------------------------------------------
constexpr int kW1Stride = kFeat + 8, kW2Stride = kHid + 8, kXStride = kFeat + 8;
// warps of a block that run the network: eight in the grid-wide placement
// kernel; four inside the persistent batch kernel, which keeps its shared
// memory under 32 KB so that the L1 left to its stack is not cut
#ifdef GQM_CTA_MODE
constexpr int kInferWarpsMax = 4;
#else
constexpr int kInferWarpsMax = 8;
#endif
struct MlpWSmem {
  uint16_t w1[kHid * kW1Stride];  // [hidden][feature]
  uint16_t w2[kHid * kW2Stride];  // [hidden][hidden]
  float b1[kHid], b2[kHid], w3[kHid];
  float b3;
};
struct MlpInferTiles {
  MlpWSmem w;
  uint16_t x[kInferWarpsMax][32 * kXStride];  // one tile of 32 input rows per warp
};
// all threads of the block; a block barrier must follow before the weights are read
__device__ inline void mlp_stage(const MlpDev &P, MlpWSmem &W) {
  for (int i = (int)threadIdx.x; i < kHid * kFeat; i += (int)blockDim.x)
    W.w1[(i / kFeat) * kW1Stride + i % kFeat] = P.w1[i];
  for (int i = (int)threadIdx.x; i < kHid * kHid; i += (int)blockDim.x)
    W.w2[(i / kHid) * kW2Stride + i % kHid] = P.w2[i];
  for (int i = (int)threadIdx.x; i < kHid; i += (int)blockDim.x) {
    W.b1[i] = P.b1[i];
    W.b2[i] = P.b2[i];
    W.w3[i] = bf2f(P.w3[i]);
  }
  if (threadIdx.x == 0) W.b3 = P.b3[0];
}
// row r of a warp's input tile (lane r writes its own row)
__device__ inline void mlp_put_row(uint16_t *x, int r, const float *f) {
  uint32_t *row = reinterpret_cast<uint32_t *>(x + r * kXStride);
  for (int j = 0; j < kFeat / 2; ++j) row[j] = (uint32_t)f2bf(f[2 * j]) | ((uint32_t)f2bf(f[2 * j + 1]) << 16);
}
#ifndef GQM_HOST_EMU
__device__ __forceinline__ uint32_t lds32(const uint16_t *p) { return *reinterpret_cast<const uint32_t *>(p); }
__device__ __forceinline__ void mma_bf16_16816(float *d, const uint32_t *a, uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
__device__ __forceinline__ uint16_t relu_bf(float v) { return f2bf(v > 0.0f ? v : 0.0f); }
// Network output for the 32 rows of tile x (row r = lane r); called by all 32
// lanes of a warp.
__device__ inline float mlp_forward_regs(const MlpWSmem &W, const uint16_t *x) {
  const int lane = (int)(threadIdx.x & 31u), g = lane >> 2, q = lane & 3;
  float ys[2][2];  // [16-row block][row g, row g + 8]: the quad's layer-3 sums
#pragma unroll
  for (int ib = 0; ib < 2; ++ib) {
    const uint16_t *xr = x + (ib * 16) * kXStride;
    float c1[8][4];
#pragma unroll
    for (int j = 0; j < 8; ++j) c1[j][0] = c1[j][1] = c1[j][2] = c1[j][3] = 0.0f;
#pragma unroll
    for (int k0 = 0; k0 < kFeat; k0 += 16) {
      uint32_t a[4];
      a[0] = lds32(xr + g * kXStride + k0 + 2 * q);
      a[1] = lds32(xr + (g + 8) * kXStride + k0 + 2 * q);
      a[2] = lds32(xr + g * kXStride + k0 + 2 * q + 8);
      a[3] = lds32(xr + (g + 8) * kXStride + k0 + 2 * q + 8);
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const uint16_t *b = W.w1 + (8 * j + g) * kW1Stride + k0 + 2 * q;
        mma_bf16_16816(c1[j], a, lds32(b), lds32(b + 8));
      }
    }
    uint32_t a2[4][4];
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
      const int ca = 16 * kk + 2 * q, cb = ca + 8;
      const float *u = c1[2 * kk], *v = c1[2 * kk + 1];
      a2[kk][0] = (uint32_t)relu_bf(u[0] + W.b1[ca]) | ((uint32_t)relu_bf(u[1] + W.b1[ca + 1]) << 16);
      a2[kk][1] = (uint32_t)relu_bf(u[2] + W.b1[ca]) | ((uint32_t)relu_bf(u[3] + W.b1[ca + 1]) << 16);
      a2[kk][2] = (uint32_t)relu_bf(v[0] + W.b1[cb]) | ((uint32_t)relu_bf(v[1] + W.b1[cb + 1]) << 16);
      a2[kk][3] = (uint32_t)relu_bf(v[2] + W.b1[cb]) | ((uint32_t)relu_bf(v[3] + W.b1[cb + 1]) << 16);
    }
    float c2[8][4];
#pragma unroll
    for (int j = 0; j < 8; ++j) c2[j][0] = c2[j][1] = c2[j][2] = c2[j][3] = 0.0f;
#pragma unroll
    for (int kk = 0; kk < 4; ++kk)
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const uint16_t *b = W.w2 + (8 * j + g) * kW2Stride + 16 * kk + 2 * q;
        mma_bf16_16816(c2[j], a2[kk], lds32(b), lds32(b + 8));
      }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      float sum = 0.0f;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int c = 8 * j + 2 * q;
        sum += bf2f(relu_bf(c2[j][2 * h] + W.b2[c])) * W.w3[c];
        sum += bf2f(relu_bf(c2[j][2 * h + 1] + W.b2[c + 1])) * W.w3[c + 1];
      }
      sum += __shfl_xor_sync(0xffffffffu, sum, 1);
      sum += __shfl_xor_sync(0xffffffffu, sum, 2);
      ys[ib][h] = sum;
    }
  }
  // row r = lane: block r / 16, half (r % 16) / 8, held by the quad of lane 4 (r % 8)
  const int src = 4 * (lane & 7);
  const float y00 = __shfl_sync(0xffffffffu, ys[0][0], src), y01 = __shfl_sync(0xffffffffu, ys[0][1], src);
  const float y10 = __shfl_sync(0xffffffffu, ys[1][0], src), y11 = __shfl_sync(0xffffffffu, ys[1][1], src);
  const bool hi = (lane >> 3) & 1;
  return W.b3 + ((lane >> 4) ? (hi ? y11 : y10) : (hi ? y01 : y00));
}
#endif

// ---------------------------------------------------------------------------
// Features of a bad triangle (scale free, bounded to [-20, 20]): angles, log
// edge ratios, the circumcenter's position on the bisector (log and asinh),
// the neighbours' shapes and apex positions (asinh), subsegment flags and the
// distance to the nearest subsegment over the shortest edge (at most 10).  The triangle is taken with its shortest edge first
// (org, dest) and the apex opposite it, as computeCircumcenter does.
// ---------------------------------------------------------------------------
__device__ inline double tri_angle(double2 p, double2 a, double2 b) {  // angle at p
  const double ux = a.x - p.x, uy = a.y - p.y, vx = b.x - p.x, vy = b.y - p.y;
  return atan2(fabs(ux * vy - uy * vx), ux * vx + uy * vy);
}
__device__ inline double seg_dist(double2 p, double2 a, double2 b) {
  const double dx = b.x - a.x, dy = b.y - a.y, l2 = dx * dx + dy * dy;
  double t = l2 > 0 ? ((p.x - a.x) * dx + (p.y - a.y) * dy) / l2 : 0.0;
  t = t < 0 ? 0 : (t > 1 ? 1 : t);
  const double ex = a.x + t * dx - p.x, ey = a.y + t * dy - p.y;
  return sqrt(ex * ex + ey * ey);
}
// Geometry of the learned placement for triangle t: the shortest edge's
// vertices o, d (edge index e), apex a, and the bisector positions.
struct Bisector {
  int e;            // edge index (opposite vertex) of the shortest edge
  double2 o, d, a;  // org, dest of the shortest edge, apex
  double len;       // shortest edge length
  double2 mid, nrm; // edge midpoint, unit normal towards the apex side
  double s_cc;      // circumcenter's position along the bisector, in edge lengths
};
__device__ inline Bisector bisector_of(const Mesh &M, int t) {
  const int4 v = M.tv[t];
  const double2 p[3] = {M.pts[v.x], M.pts[v.y], M.pts[v.z]};
  double l[3];
  for (int i = 0; i < 3; ++i) {
    const double2 a = p[(i + 1) % 3], b = p[(i + 2) % 3];
    l[i] = (a.x - b.x) * (a.x - b.x) + (a.y - b.y) * (a.y - b.y);
  }
  int e = 0;
  if (l[1] < l[e]) e = 1;
  if (l[2] < l[e]) e = 2;
  Bisector B;
  B.e = e;
  B.o = p[(e + 1) % 3];
  B.d = p[(e + 2) % 3];
  B.a = p[e];
  B.len = sqrt(l[e]);
  B.mid = make_double2(0.5 * (B.o.x + B.d.x), 0.5 * (B.o.y + B.d.y));
  // counterclockwise triangle: the apex is left of o -> d
  B.nrm = make_double2(-(B.d.y - B.o.y) / B.len, (B.d.x - B.o.x) / B.len);
  // circumcenter: on the bisector at distance sqrt(R^2 - len^2/4) (apex side
  // when the apex angle is acute)
  const double area2 = (B.d.x - B.o.x) * (B.a.y - B.o.y) - (B.d.y - B.o.y) * (B.a.x - B.o.x);
  const double la = sqrt(l[(e + 1) % 3]), lb = sqrt(l[(e + 2) % 3]);
  const double R = B.len * la * lb / (2.0 * fabs(area2));
  double h = R * R - 0.25 * B.len * B.len;
  h = h > 0 ? sqrt(h) : 0.0;
  const double cosA = ((B.o.x - B.a.x) * (B.d.x - B.a.x) + (B.o.y - B.a.y) * (B.d.y - B.a.y));
  B.s_cc = (cosA >= 0 ? h : -h) / B.len;
  return B;
}
__device__ inline void features_of(const Mesh &M, int t, const Bisector &B, double offc, float *f) {
  const int4 v = M.tv[t], nb = M.tn[t], sg = M.tsg[t];
  const double2 p[3] = {M.pts[v.x], M.pts[v.y], M.pts[v.z]};
  int k = 0;
  const int e = B.e;
  // own angles (apex, org, dest) and edge ratios
  f[k++] = (float)tri_angle(B.a, B.o, B.d);
  f[k++] = (float)tri_angle(B.o, B.d, B.a);
  f[k++] = (float)tri_angle(B.d, B.a, B.o);
  const double lo = sqrt((B.a.x - B.d.x) * (B.a.x - B.d.x) + (B.a.y - B.d.y) * (B.a.y - B.d.y)) / B.len;
  const double ld = sqrt((B.a.x - B.o.x) * (B.a.x - B.o.x) + (B.a.y - B.o.y) * (B.a.y - B.o.y)) / B.len;
  f[k++] = (float)log(lo);
  f[k++] = (float)log(ld);
  f[k++] = (float)log(B.s_cc > 1e-12 ? B.s_cc : 1e-12);
  f[k++] = (float)offc;
  f[k++] = (float)asinh(B.s_cc - offc);
  f[k++] = (float)M.gc2;
  // neighbours across the three edges, shortest edge first
  double dmin = 10.0;
  for (int r = 0; r < 3; ++r) {
    const int i = (e + r) % 3;
    const int o = comp(nb, i);
    const int s = comp(sg, i);
    f[k++] = s >= 0 ? 1.0f : 0.0f;
    if (s >= 0) dmin = fmin(dmin, seg_dist(B.mid, p[(i + 1) % 3], p[(i + 2) % 3]) / B.len);
    if (o < 0) {
      f[k++] = 0.0f;
      f[k++] = 0.0f;
      f[k++] = 0.0f;
      f[k++] = 0.0f;
      continue;
    }
    const int nt = dtri(o), ni = dori(o);
    const int4 w = M.tv[nt];
    const double2 q[3] = {M.pts[w.x], M.pts[w.y], M.pts[w.z]};
    const double a0 = tri_angle(q[0], q[1], q[2]), a1 = tri_angle(q[1], q[2], q[0]), a2 = tri_angle(q[2], q[0], q[1]);
    f[k++] = (float)fmin(a0, fmin(a1, a2));
    f[k++] = (float)tri_angle(q[ni], q[(ni + 1) % 3], q[(ni + 2) % 3]);  // opposite the shared edge
    const double2 x = q[ni];
    f[k++] = (float)asinh(((x.x - B.mid.x) * B.nrm.x + (x.y - B.mid.y) * B.nrm.y) / B.len);
    f[k++] = (float)asinh(((x.x - B.mid.x) * (B.d.x - B.o.x) + (x.y - B.mid.y) * (B.d.y - B.o.y)) / (B.len * B.len));
    const int4 ns = M.tsg[nt];
    for (int j = 0; j < 3; ++j) {
      const int s2 = comp(ns, j);
      if (s2 >= 0) dmin = fmin(dmin, seg_dist(B.mid, q[(j + 1) % 3], q[(j + 2) % 3]) / B.len);
    }
  }
  f[k++] = (float)dmin;
  while (k < kFeat - 1) f[k++] = 0.0f;
  f[kFeat - 1] = 1.0f;
  for (int j = 0; j < kFeat; ++j) f[j] = fminf(20.0f, fmaxf(-20.0f, f[j]));  // bounded inputs
}

// Does point c encroach (diametral circle, Ruppert) a subsegment on the edges
// of triangle t or of its neighbours?
__device__ inline bool encroaches_near(const Mesh &M, int t, double2 c) {
  const int4 nb = M.tn[t];
  for (int r = -1; r < 3; ++r) {
    const int u = r < 0 ? t : dtri(comp(nb, r));
    if (u < 0) continue;
    const int4 v = M.tv[u], sg = M.tsg[u];
    const double2 p[3] = {M.pts[v.x], M.pts[v.y], M.pts[v.z]};
    for (int j = 0; j < 3; ++j) {
      if (comp(sg, j) < 0) continue;
      const double2 a = p[(j + 1) % 3], b = p[(j + 2) % 3];
      if ((a.x - c.x) * (b.x - c.x) + (a.y - c.y) * (b.y - c.y) < 0.0) return true;
    }
  }
  return false;
}

}  // namespace gqm
