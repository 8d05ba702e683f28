// Test-only stand-in for the CUDA runtime, used to compile the refiner's own
// sources (gpu_cdt_refine_b200/csrc/refine.cu) as host C++ so that their index
// arithmetic and results can be checked on a machine without a GPU.  Kernels
// run as ordinary functions with one thread covering every element of its
// grid-stride loop.  Never linked into the product library.
#pragma once
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>

#define GQM_HOST_EMU 1
#define __global__
#define __device__
#define __host__
#define __forceinline__ inline
#define __noinline__
#define __shared__ static thread_local
#define __launch_bounds__(...)
#define __align__(n) __attribute__((aligned(n)))

struct dim3_emu {
  unsigned x, y, z;
};
static dim3_emu threadIdx = {0, 0, 0}, blockIdx = {0, 0, 0}, blockDim = {1, 1, 1}, gridDim = {1, 1, 1};

struct int2 {
  int x, y;
};
struct int4 {
  int x, y, z, w;
};
struct double2 {
  double x, y;
};
inline int4 make_int4(int a, int b, int c, int d) { return int4{a, b, c, d}; }
inline int2 make_int2(int a, int b) { return int2{a, b}; }
inline double2 make_double2(double a, double b) { return double2{a, b}; }
using std::max;
using std::min;

inline int atomicMin(int *a, int v) {
  int o = *a;
  if (v < o) *a = v;
  return o;
}
inline int atomicMax(int *a, int v) {
  int o = *a;
  if (v > o) *a = v;
  return o;
}
inline unsigned long long atomicMax(unsigned long long *a, unsigned long long v) {
  unsigned long long o = *a;
  if (v > o) *a = v;
  return o;
}
inline unsigned long long atomicMin(unsigned long long *a, unsigned long long v) {
  unsigned long long o = *a;
  if (v < o) *a = v;
  return o;
}
inline unsigned atomicAdd(unsigned *a, unsigned v) {
  unsigned o = *a;
  *a += v;
  return o;
}
inline void __threadfence() {}
inline unsigned atomicOr(unsigned *a, unsigned v) {
  unsigned o = *a;
  *a |= v;
  return o;
}
inline unsigned atomicAnd(unsigned *a, unsigned v) {
  unsigned o = *a;
  *a &= v;
  return o;
}
inline unsigned long long atomicCAS(unsigned long long *a, unsigned long long c, unsigned long long v) {
  unsigned long long o = *a;
  if (o == c) *a = v;
  return o;
}
inline unsigned __int128 atomicCAS(unsigned __int128 *a, unsigned __int128 c, unsigned __int128 v) {
  unsigned __int128 o = *a;
  if (o == c) *a = v;
  return o;
}
inline int atomicCAS(int *a, int c, int v) {
  int o = *a;
  if (o == c) *a = v;
  return o;
}
inline unsigned long long atomicAdd(unsigned long long *a, unsigned long long v) {
  unsigned long long o = *a;
  *a += v;
  return o;
}
inline int atomicExch(int *a, int v) {
  int o = *a;
  *a = v;
  return o;
}
inline unsigned long long atomicExch(unsigned long long *a, unsigned long long v) {
  unsigned long long o = *a;
  *a = v;
  return o;
}
inline int atomicAdd(int *a, int v) {
  int o = *a;
  *a += v;
  return o;
}
inline void __syncthreads() {}
inline void __syncwarp(unsigned = 0xffffffffu) {}
inline int __shfl_down_sync(unsigned, int v, int) { return v; }
inline unsigned __ballot_sync(unsigned, bool p) { return p ? 1u : 0u; }
inline unsigned __activemask() { return 1u; }
inline int __popc(unsigned v) { return __builtin_popcount(v); }
inline int __shfl_up_sync(unsigned, int v, int) { return v; }
inline int __shfl_sync(unsigned, int v, int) { return v; }
inline int __ffs(unsigned v) { return __builtin_ffs(v); }
inline unsigned __match_any_sync(unsigned, int) { return 1u; }
inline int __clz(int v) { return v == 0 ? 32 : __builtin_clz((unsigned)v); }

typedef int cudaError_t;
typedef void *cudaStream_t;
typedef std::chrono::steady_clock::time_point *cudaEvent_t;
enum { cudaSuccess = 0, cudaErrorMemoryAllocation = 2 };
enum cudaMemcpyKind { cudaMemcpyHostToDevice, cudaMemcpyDeviceToHost, cudaMemcpyDeviceToDevice };
#define cudaStreamNonBlocking 1

// Fault injection for the CPU tests: allocation number `fail_at` (counted
// from the last gqm_fake_fail_alloc_at call, device and pinned allocations
// together) fails as an out-of-memory would; -1 turns it off.
inline long long g_fake_fail_at = -1;
inline long long g_fake_allocs = 0;
extern "C" __attribute__((weak)) void gqm_fake_fail_alloc_at(long long fail_at) {
  g_fake_fail_at = fail_at;
  g_fake_allocs = 0;
}
extern "C" __attribute__((weak)) long long gqm_fake_alloc_count(void) { return g_fake_allocs; }
inline cudaError_t cudaMalloc(void **p, size_t n) {
  if (g_fake_allocs++ == g_fake_fail_at) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  *p = calloc(1, n ? n : 1);
  return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
inline cudaError_t cudaMallocHost(void **p, size_t n) { return cudaMalloc(p, n); }
inline cudaError_t cudaFree(void *p) {
  free(p);
  return cudaSuccess;
}
inline cudaError_t cudaFreeHost(void *p) { return cudaFree(p); }
inline cudaError_t cudaMemcpyAsync(void *d, const void *s, size_t n, cudaMemcpyKind, cudaStream_t = nullptr) {
  memmove(d, s, n);
  return cudaSuccess;
}
inline cudaError_t cudaMemcpy(void *d, const void *s, size_t n, cudaMemcpyKind k) { return cudaMemcpyAsync(d, s, n, k); }
inline cudaError_t cudaMemset(void *d, int v, size_t n) {
  memset(d, v, n);
  return cudaSuccess;
}
inline cudaError_t cudaMemsetAsync(void *d, int v, size_t n, cudaStream_t = nullptr) {
  memset(d, v, n);
  return cudaSuccess;
}
inline cudaError_t cudaStreamCreateWithFlags(cudaStream_t *s, int) {
  *s = (void *)1;
  return cudaSuccess;
}
inline cudaError_t cudaStreamDestroy(cudaStream_t) { return cudaSuccess; }
inline cudaError_t cudaStreamSynchronize(cudaStream_t) { return cudaSuccess; }
inline cudaError_t cudaSetDevice(int) { return cudaSuccess; }
inline cudaError_t cudaGetDeviceCount(int *n) {
  *n = 1;
  return cudaSuccess;
}
inline cudaError_t cudaEventCreate(cudaEvent_t *e) {
  *e = new std::chrono::steady_clock::time_point();
  return cudaSuccess;
}
inline cudaError_t cudaEventDestroy(cudaEvent_t e) {
  delete e;
  return cudaSuccess;
}
inline cudaError_t cudaEventRecord(cudaEvent_t e, cudaStream_t = nullptr) {
  *e = std::chrono::steady_clock::now();
  return cudaSuccess;
}
inline cudaError_t cudaEventElapsedTime(float *ms, cudaEvent_t a, cudaEvent_t b) {
  *ms = std::chrono::duration<float, std::milli>(*b - *a).count();
  return cudaSuccess;
}
inline cudaError_t cudaGetLastError() { return cudaSuccess; }
inline const char *cudaGetErrorString(cudaError_t) { return "emulated"; }
template <class T>
inline cudaError_t cudaMemcpyToSymbolAsync(T &sym, const void *src, size_t n, size_t off, cudaMemcpyKind,
                                           cudaStream_t = nullptr) {
  memcpy((char *)&sym + off, src, n);
  return cudaSuccess;
}
template <class T>
inline cudaError_t cudaMemcpyFromSymbol(void *dst, const T &sym, size_t n) {
  memcpy(dst, &sym, n);
  return cudaSuccess;
}
template <class T>
inline cudaError_t cudaGetSymbolAddress(void **p, T &sym) {
  *p = (void *)&sym;
  return cudaSuccess;
}
typedef void *cudaGraph_t;
typedef int cudaGraphConditionalHandle;
typedef void *cudaGraphExec_t;
inline cudaError_t cudaGraphLaunch(cudaGraphExec_t, cudaStream_t) { return 1; }
