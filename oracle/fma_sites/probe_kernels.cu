// Runs three of the reference's own kernels (GPU_Refine/refine.cu, linked from
// the reference's sources and compiled as its project compiles them: nvcc's
// default contraction) on 100,000 random inputs each, and writes inputs and
// outputs for analyze.py:
//   kernelComputeCircumcenter  off-centers with offConstant 3 and 2 (half of
//                              the triangles skinny, so the off-center is taken),
//                              then circumcenters
//   kernelMarkBadTriangles     isosceles triangles whose apex angle is 20 deg
//                              to within 1e-14, the apex in each vertex position
//   kernelMarkAllEncsegs       apex angles at the Chew lens boundary and at the
//                              right angle to within 1e-14 (both modes)
// Every index stays inside the arrays: triangle i is vertices 3i..3i+2 with no
// neighbour and no subsegment, subsegment i lies on edge 0 of triangle i.
// Build: make -C oracle fma-probes.  Run on a GPU: fma_probe_kernels OUT.bin
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <random>
#include <vector>
#include "refine.h"

__global__ void kernelComputeCircumcenter(REAL2 *, int *, int *, int, REAL2 *, int *, REAL, bool);
__global__ void kernelMarkBadTriangles(REAL2 *, PStatus *, int *, int *, int *, int *, int *, TStatus *, int *, int, REAL);
__global__ void kernelMarkAllEncsegs(REAL2 *, int *, int *, int *, int *, int, int, REAL);

template <class T> T *up(const std::vector<T> &h) {
  T *d = nullptr;
  cudaMalloc(&d, sizeof(T) * h.size());
  cudaMemcpy(d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice);
  return d;
}
template <class T> void down(std::vector<T> &h, const T *d) { cudaMemcpy(h.data(), d, sizeof(T) * h.size(), cudaMemcpyDeviceToHost); }

int main(int argc, char **argv) {
  const int n = 100000;
  std::mt19937_64 g(11);
  std::uniform_real_distribution<double> U(0.0, 1000.0), A(0.0, 6.283185307179586), L(0.5, 50.0), E(-1e-14, 1e-14), R(1.0, 1.5), S(0.05, 0.3);
  FILE *f = fopen(argv[1], "wb");
  std::vector<int> tri(3 * n), act(n), nbr(3 * n, -1), t2s(3 * n, -1), s2s(n, 0), segl(2 * n, 0);
  for (int i = 0; i < 3 * n; ++i) tri[i] = i;
  for (int i = 0; i < n; ++i) act[i] = i;
  int *dtri = up(tri), *dact = up(act), *dnbr = up(nbr), *dt2s = up(t2s), *ds2s = up(s2s), *dsegl = up(segl);
  // 1. circumcenters of random triangles (CCW)
  {
    std::vector<double2> p(3 * n);
    for (int i = 0; i < n; ++i) {
      double2 a = make_double2(U(g), U(g)), b = make_double2(U(g), U(g)), c = make_double2(U(g), U(g));
      if (i & 1) {  // a skinny triangle: apex angle 3-17 degrees at a, legs of similar length
        double r = A(g), l1 = L(g), l2 = l1 * R(g), t = S(g);
        b = make_double2(a.x + l1 * cos(r), a.y + l1 * sin(r));
        c = make_double2(a.x + l2 * cos(r + t), a.y + l2 * sin(r + t));
        if (i & 2) std::swap(a, b), std::swap(b, c);  // rotate the vertex order
      }
      double o = (b.x - a.x) * (c.y - a.y) - (b.y - a.y) * (c.x - a.x);
      if (o < 0) std::swap(b, c);
      p[3 * i] = a; p[3 * i + 1] = b; p[3 * i + 2] = c;
    }
    double2 *dp = up(p);
    std::vector<double2> cc(n);
    std::vector<int> pr(n);
    double2 *dcc = up(cc);
    int *dpr = up(pr);
    fwrite(p.data(), sizeof(double2), 3 * n, f);
    for (int mode = 0; mode < 3; ++mode) {  // off-centers with offConstant 3 and 2, then circumcenters
      kernelComputeCircumcenter<<<(n + 255) / 256, 256>>>(dp, dtri, dact, n, dcc, dpr, mode == 0 ? 3.0 : 2.0,
                                                          mode < 2);
      down(cc, dcc);
      fwrite(cc.data(), sizeof(double2), n, f);
    }
  }
  // 2. bad-triangle test near theta = 20 deg: apex angle 20 deg (+ tiny), random legs
  {
    std::vector<double2> p(3 * n);
    const double th = 20.0 * 3.141592653589793 / 180.0;
    for (int i = 0; i < n; ++i) {
      double2 a = make_double2(U(g), U(g));
      double r = A(g), l1 = L(g), l2 = l1 * R(g), t = th * (1.0 + E(g));
      double2 b = make_double2(a.x + l1 * cos(r), a.y + l1 * sin(r));
      double2 c = make_double2(a.x + l2 * cos(r + t), a.y + l2 * sin(r + t));
      // CCW: c is at +t from b; the apex (smallest angle) goes to position i % 3
      if (i % 3 == 0) { p[3 * i] = a; p[3 * i + 1] = b; p[3 * i + 2] = c; }
      else if (i % 3 == 1) { p[3 * i] = c; p[3 * i + 1] = a; p[3 * i + 2] = b; }
      else { p[3 * i] = b; p[3 * i + 1] = c; p[3 * i + 2] = a; }
    }
    double2 *dp = up(p);
    std::vector<PStatus> ps(3 * n);
    std::vector<TStatus> ts(n);
    for (auto &s : ts) s._status = 4;  // check
    PStatus *dps = up(ps);
    TStatus *dts = up(ts);
    kernelMarkBadTriangles<<<(n + 255) / 256, 256>>>(dp, dps, dtri, dnbr, dsegl, ds2s, dt2s, dts, dact, n, 20.0);
    down(ts, dts);
    fwrite(p.data(), sizeof(double2), 3 * n, f);
    fwrite(ts.data(), 1, n, f);
  }
  // 3. encroachment: apex near the right angle (Ruppert) or near the lens (Chew); triangle (apex, org, dest)
  for (int mode = 0; mode < 2; ++mode) {
    std::vector<double2> p(3 * n);
    const double gc = cos(20.0 * 3.141592653589793 / 180.0);
    const double lens = mode ? 3.141592653589793 / 2 : acos(-(2 * gc * gc - 1));  // apex angle at the boundary
    for (int i = 0; i < n; ++i) {
      double2 a = make_double2(U(g), U(g));
      double r = A(g), l1 = L(g), l2 = L(g), t = lens * (1.0 + E(g));
      double2 o = make_double2(a.x + l1 * cos(r), a.y + l1 * sin(r));
      double2 d = make_double2(a.x + l2 * cos(r - t), a.y + l2 * sin(r - t));
      p[3 * i] = a; p[3 * i + 1] = o; p[3 * i + 2] = d;
    }
    std::vector<int> s2t(n), enc(n);
    for (int i = 0; i < n; ++i) s2t[i] = i << 2;  // edge 0 of triangle i: org = v1, dest = v2, apex = v0
    double2 *dp = up(p);
    int *ds2t = up(s2t), *denc = up(enc);
    kernelMarkAllEncsegs<<<(n + 255) / 256, 256>>>(dp, dtri, dnbr, ds2t, denc, n, mode, 20.0);
    down(enc, denc);
    fwrite(p.data(), sizeof(double2), 3 * n, f);
    fwrite(enc.data(), sizeof(int), n, f);
  }
  fclose(f);
  cudaError_t e = cudaDeviceSynchronize();
  printf("probe2 %s\n", cudaGetErrorString(e));
  return e == cudaSuccess ? 0 : 1;
}
