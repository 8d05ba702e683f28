// Linux command-line driver for the reference GPU refiner (test oracle only).
//
// The reference ships a Windows/GLUT console program (GPU_Refine/main.cpp) that
// calls GPU_Refine_Quality at main.cpp:1863.  That file does not build on Linux,
// so this driver takes its place: it reads a CDT in the binary "GQMCDT1" format
// (written by gpu_cdt_refine_b200.cdtio), calls the reference entry point
// GPU_Refine_Quality (GPU_Refine/refine.h:385-386) unmodified, and writes the
// refined CDT back in the same format.  Timing mirrors main.cpp:1858-1868: the
// wall time of the whole call, host copies included.
//
// Usage: gqm_ref_run IN OUT THETA POLICY MODE [REPS]
//   POLICY 0 = Circumcenter, 1 = Offcenter   (refine.h:32)
//   MODE   1 = Ruppert, 0 = Chew              (refine.cu:131)
// A JSON summary line prefixed with "GQMREF " is printed on stderr.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <chrono>
#include <vector>
#include "refine.h"

static bool read_cdt(const char *path, triangulateio *io) {
  FILE *f = fopen(path, "rb");
  if (!f) return false;
  char magic[8];
  int hdr[4];
  if (fread(magic, 1, 8, f) != 8 || memcmp(magic, "GQMCDT1", 7) != 0) { fclose(f); return false; }
  if (fread(hdr, sizeof(int), 4, f) != 4) { fclose(f); return false; }
  memset(io, 0, sizeof(*io));
  io->numberofpoints = hdr[0];
  io->numberoftriangles = hdr[1];
  io->numberofsegments = hdr[2];
  io->numberofcorners = 3;
  io->pointlist = new double[2 * (size_t)hdr[0]];
  io->trianglelist = new int[3 * (size_t)hdr[1]];
  io->neighborlist = new int[3 * (size_t)hdr[1]];
  io->segmentlist = new int[2 * (size_t)hdr[2] + 2];
  bool ok = fread(io->pointlist, sizeof(double), 2 * (size_t)hdr[0], f) == 2 * (size_t)hdr[0];
  ok = ok && fread(io->trianglelist, sizeof(int), 3 * (size_t)hdr[1], f) == 3 * (size_t)hdr[1];
  if (hdr[3]) ok = ok && fread(io->neighborlist, sizeof(int), 3 * (size_t)hdr[1], f) == 3 * (size_t)hdr[1];
  ok = ok && fread(io->segmentlist, sizeof(int), 2 * (size_t)hdr[2], f) == 2 * (size_t)hdr[2];
  fclose(f);
  return ok && hdr[3] == 1;
}

static bool write_cdt(const char *path, const triangulateio *io) {
  FILE *f = fopen(path, "wb");
  if (!f) return false;
  const char magic[8] = {'G', 'Q', 'M', 'C', 'D', 'T', '1', 0};
  int hdr[4] = {io->numberofpoints, io->numberoftriangles, io->numberofsegments, 1};
  fwrite(magic, 1, 8, f);
  fwrite(hdr, sizeof(int), 4, f);
  fwrite(io->pointlist, sizeof(double), 2 * (size_t)io->numberofpoints, f);
  fwrite(io->trianglelist, sizeof(int), 3 * (size_t)io->numberoftriangles, f);
  fwrite(io->neighborlist, sizeof(int), 3 * (size_t)io->numberoftriangles, f);
  fwrite(io->segmentlist, sizeof(int), 2 * (size_t)io->numberofsegments, f);
  fclose(f);
  return true;
}

int main(int argc, char **argv) {
  if (argc < 6) {
    fprintf(stderr, "usage: %s IN OUT THETA POLICY MODE [REPS]\n", argv[0]);
    return 2;
  }
  triangulateio in;
  if (!read_cdt(argv[1], &in)) {
    fprintf(stderr, "cannot read %s\n", argv[1]);
    return 2;
  }
  double theta = atof(argv[3]);
  InsertPolicy pol = atoi(argv[4]) ? Offcenter : Circumcenter;
  int mode = atoi(argv[5]);
  int reps = argc > 6 ? atoi(argv[6]) : 1;
  if (reps < 1) reps = 1;

  cudaFree(0);  // context creation outside the timed region
  std::vector<double> times;
  triangulateio out;
  for (int r = 0; r < reps; ++r) {
    memset(&out, 0, sizeof(out));
    cudaDeviceSynchronize();
    auto t0 = std::chrono::steady_clock::now();
    GPU_Refine_Quality(&in, &out, theta, pol, Connected, mode, -1, NULL, NULL);
    cudaDeviceSynchronize();
    auto t1 = std::chrono::steady_clock::now();
    times.push_back(std::chrono::duration<double, std::milli>(t1 - t0).count());
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
      fprintf(stderr, "cuda error %s\n", cudaGetErrorString(e));
      return 3;
    }
    if (r + 1 < reps) {
      delete[] out.pointlist;
      delete[] out.trianglelist;
      delete[] out.neighborlist;
      delete[] out.segmentlist;
    }
  }
  if (!write_cdt(argv[2], &out)) {
    fprintf(stderr, "cannot write %s\n", argv[2]);
    return 2;
  }
  fprintf(stderr, "GQMREF {\"points\": %d, \"triangles\": %d, \"segments\": %d, \"ms\": [", out.numberofpoints,
          out.numberoftriangles, out.numberofsegments);
  for (size_t i = 0; i < times.size(); ++i) fprintf(stderr, "%s%.3f", i ? ", " : "", times[i]);
  fprintf(stderr, "]}\n");
  return 0;
}
