// Evaluates the reference's predicates (GPU_Refine/cudaCCW.h, included from the
// reference's sources and compiled as its project compiles them: nvcc's default
// contraction) on 200,000 random quadruples, the first three points nearly
// collinear; writes the inputs and the four results per quadruple (cuda_ccw,
// cuda_fast, cuda_inCircle, cuda_inCircle_exact) for analyze.py.
// Build: make -C oracle fma-probes.  Run on a GPU: fma_probe_predicates OUT.bin
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>
#define REAL double
#define REAL2 double2
double hostConst[13];
#include "cudaCCW.h"
__global__ void probe(const double2 *p, int n, double *o) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double2 a = p[4 * i], b = p[4 * i + 1], c = p[4 * i + 2], d = p[4 * i + 3];
  o[4 * i] = cuda_ccw(a, b, c);
  o[4 * i + 1] = cuda_fast(a, b, c);
  o[4 * i + 2] = cuda_inCircle(a, b, c, d);
  o[4 * i + 3] = cuda_inCircle_exact(a, b, c, d);
}
int main(int argc, char **argv) {
  int n = 200000;
  std::mt19937_64 g(7);
  std::uniform_real_distribution<double> U(0.0, 1000.0), J(-1e-3, 1e-3);
  std::vector<double2> h(4 * n);
  for (int i = 0; i < n; ++i) {
    // a, b, c nearly collinear; d nearly on the circle of a, b, c for half of them
    double ax = U(g), ay = U(g), bx = U(g), by = U(g), t = U(g) / 1000.0;
    double cx = ax + t * (bx - ax) + J(g), cy = ay + t * (by - ay) + J(g);
    h[4 * i] = make_double2(ax, ay);
    h[4 * i + 1] = make_double2(bx, by);
    h[4 * i + 2] = make_double2(cx, cy);
    h[4 * i + 3] = make_double2(U(g), U(g));
  }
  double2 *dp; double *dout;
  cudaMalloc(&dp, sizeof(double2) * 4 * n);
  cudaMalloc(&dout, sizeof(double) * 4 * n);
  cudaMemcpy(dp, h.data(), sizeof(double2) * 4 * n, cudaMemcpyHostToDevice);
  probe<<<(n + 255) / 256, 256>>>(dp, n, dout);
  std::vector<double> o(4 * n);
  if (cudaMemcpy(o.data(), dout, sizeof(double) * 4 * n, cudaMemcpyDeviceToHost) != cudaSuccess) return 1;
  FILE *f = fopen(argv[1], "wb");
  fwrite(h.data(), sizeof(double2), 4 * n, f);
  fwrite(o.data(), sizeof(double), 4 * n, f);
  fclose(f);
  printf("probe ok %d\n", n);
  return 0;
}
