// Link-time launch interposer for the traced reference build (test oracle only).
//
// Same empty-grid guard as launch_guard.cpp, plus a step trace: at every
// launch of kernelCheckFlipping (GPU_Refine/refine.cu:778), i.e. at the start
// of every flip step, the mesh arrays it receives are copied to the host and
// one line of FNV-1a digests is written to the file named by GQM_REF_TRACE:
//
//   F <step> nt=<triangles> nact=<active> tri= nbr= t2s= ts= act= np=<points> pts= mesh=
//
// The oracle writes the same line at the same point (gqm_oracle_trace), so the
// two traces show the first flip step at which two runs part.  "mesh" digests
// the live triangles as a set (each rotated to its smallest vertex, sorted),
// which is independent of the slots the triangles occupy.
//
// The argument layout read here is kernelCheckFlipping's parameter list:
// (pointlist, PStatus, trianglelist, neighborlist, tri2subseg, TStatus,
//  flipBy, active, numberofactive); the triangle count comes from the
// preceding kernelInitFlipOri(TStatus, numberoftriangles) (refine.cu:759).
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <string>
#include <vector>

namespace {
FILE *g_out = nullptr;
bool g_init = false;
long g_step = 0;
int g_nt = 0;
std::map<const void *, int> g_kind;  // 0 other, 1 InitFlipOri, 2 CheckFlipping

unsigned long long fnv64(const void *p, size_t n) {
  const unsigned char *b = static_cast<const unsigned char *>(p);
  unsigned long long h = 1469598103934665603ULL;
  for (size_t i = 0; i < n; ++i) {
    h ^= b[i];
    h *= 1099511628211ULL;
  }
  return h;
}

int kind_of(const void *f) {
  auto it = g_kind.find(f);
  if (it != g_kind.end()) return it->second;
  const char *name = nullptr;
  int k = 0;
  if (cudaFuncGetName(&name, f) == cudaSuccess && name) {
    std::string s(name);
    if (s.find("kernelInitFlipOri") != std::string::npos) k = 1;
    if (s.find("kernelCheckFlipping") != std::string::npos) k = 2;
  }
  g_kind[f] = k;
  return k;
}

template <class T>
std::vector<T> fetch(const void *dev, size_t n) {
  std::vector<T> h(n);
  if (n) cudaMemcpy(h.data(), dev, sizeof(T) * n, cudaMemcpyDeviceToHost);
  return h;
}

void trace_step(void **args) {
  int nt = g_nt;
  const void *pts = *static_cast<void **>(args[0]);
  auto tri = fetch<int>(*static_cast<void **>(args[2]), 3L * nt);
  auto nbr = fetch<int>(*static_cast<void **>(args[3]), 3L * nt);
  auto t2s = fetch<int>(*static_cast<void **>(args[4]), 3L * nt);
  auto ts = fetch<unsigned char>(*static_cast<void **>(args[5]), nt);
  int nact = *static_cast<int *>(args[8]);
  auto act = fetch<int>(*static_cast<void **>(args[7]), nact);
  int np = 0;
  for (int v : tri) np = std::max(np, v + 1);
  auto p = fetch<double>(pts, 2L * np);
  std::vector<std::array<int, 3>> live;
  for (int t = 0; t < nt; ++t) {
    if (!(ts[t] & 1)) continue;
    int v[3] = {tri[3 * t], tri[3 * t + 1], tri[3 * t + 2]};
    int k = (v[0] <= v[1] && v[0] <= v[2]) ? 0 : (v[1] <= v[2] ? 1 : 2);
    live.push_back({v[k], v[(k + 1) % 3], v[(k + 2) % 3]});
  }
  std::sort(live.begin(), live.end());
  fprintf(g_out,
          "F %ld nt=%d nact=%d tri=%016llx nbr=%016llx t2s=%016llx ts=%016llx act=%016llx np=%d pts=%016llx "
          "mesh=%016llx\n",
          g_step++, nt, nact, fnv64(tri.data(), 12L * nt), fnv64(nbr.data(), 12L * nt), fnv64(t2s.data(), 12L * nt),
          fnv64(ts.data(), nt), fnv64(act.data(), 4L * nact), np, fnv64(p.data(), 16L * np),
          fnv64(live.data(), 12 * live.size()));
  fflush(g_out);
}
}  // namespace

extern "C" cudaError_t __real_cudaLaunchKernel(const void *func, dim3 grid, dim3 block, void **args,
                                               size_t shared, cudaStream_t stream);

extern "C" cudaError_t __wrap_cudaLaunchKernel(const void *func, dim3 grid, dim3 block, void **args,
                                               size_t shared, cudaStream_t stream) {
  if (grid.x == 0 || grid.y == 0 || grid.z == 0) return cudaSuccess;
  if (!g_init) {
    g_init = true;
    const char *path = getenv("GQM_REF_TRACE");
    if (path) g_out = fopen(path, "w");
  }
  if (g_out) {
    int k = kind_of(func);
    if (k == 1) g_nt = *static_cast<int *>(args[1]);
    if (k == 2) {
      cudaDeviceSynchronize();  // the reference runs on the legacy default stream
      trace_step(args);
    }
  }
  return __real_cudaLaunchKernel(func, grid, block, args, shared, stream);
}
