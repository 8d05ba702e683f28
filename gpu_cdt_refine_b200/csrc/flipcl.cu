// Small flip steps of the single-domain engine on one thread-block cluster.
//
// The flip-flop loop (GPU_Refine/refine.cu:2328-2490) spends most of its steps
// on small active sets.  batch.cu's k_flip_small runs such steps in one thread
// block; this kernel runs them on a cluster of 8 or 16 blocks (one per SM, up
// to 4,096 threads), so that the items of a step are spread over more warps
// and SMs while the step phases are still separated by a barrier instead of a
// launch.  The phase functions are the kernels of kernels.cuh compiled in
// cluster mode: each is a __device__ function whose grid-stride loop covers
// the cluster (the launch's grid is exactly one cluster), and a cluster
// barrier (release / acquire at cluster scope) separates consecutive phases.
//
// The phases communicate through global memory written by other SMs of the
// cluster.  This translation unit is compiled with global loads cached in L2
// only (ptxas -dlcm=cg), so no load can be served from a line that an SM's L1
// kept from before the barrier; the barrier's release / acquire orders every
// store before it with every load after it.
//
// Every step makes the same decisions as the grid kernels and the one-block
// kernel: each phase is decided by the reference's rules on the data, never by
// the thread layout.
#define GQM_CLUSTER_MODE 1
#define gqm gqm_cl
#include <cuda_runtime.h>
#ifndef GQM_HOST_EMU
#include <cooperative_groups.h>
#endif

#include <cstring>

#include "../../include/gqm_refine.h"
#include "kernels.cuh"

namespace gqm {

__device__ KTimer g_ktimer_cluster_off;

// threads per block of the cluster kernel; one block per SM
constexpr int kClusterThreads = 256;

__device__ __forceinline__ void cluster_barrier() {
#ifndef GQM_HOST_EMU
  cooperative_groups::this_cluster().sync();
#endif
}

template <int PRED>
__global__ void __launch_bounds__(kClusterThreads, 1)
    k_flip_small_cl(Mesh M, FlipCtl *fc, int *act, uint8_t *clr, int *win, int *ll, int *sl, int *fq, int *tl,
                    int limit, cudaGraphConditionalHandle h, int graph, KTimer *tm) {
  const int timed = tm->on;
  const unsigned long long start = timed ? global_ns() : 0;
  long long items = 0, wins = 0;  // the launch's work, the same in every thread (probe only)
  for (;;) {
    // Every thread reads the same two words: they were last written before
    // the barrier that ended the previous step (or by the kernel before this
    // launch), and nothing writes them until after the next barrier.
    const int nact = fc->nact;
    const int go = fc->cond && nact <= limit;
    cluster_barrier();
    if (!go) break;
    items += nact;
    FlipQ Q{fq, &fc->qn, &fc->gen};
    TouchL T{tl, &fc->tn, &fc->gen};
    k_check_flip2<PRED>(M, act, &fc->nact, clr, T, &g_ktimer_cluster_off);
    cluster_barrier();
    k_flip_winner2(M, act, &fc->nact, clr, Q, win, &fc->winn);
    cluster_barrier();
    wins += fc->winn;  // complete after the barrier; read before the next step resets it
    k_link_phase1(M, win, &fc->winn, ll, sl, &fc->epoch);
    cluster_barrier();
    k_phase2(M, win, &fc->winn, ll, sl);
    cluster_barrier();
    k_phase3q(M, win, &fc->winn, sl, Q);
    cluster_barrier();
    k_mark_red_steiner_q(M, tl, &fc->tn, Q);
    cluster_barrier();
    k_flip_reset_filter(M, tl, &fc->tn, fq, &fc->qn, act, &fc->nact_next);
    cluster_barrier();
    if (GQM_BLOCK0 && threadIdx.x == 0) {
      fc->nact = fc->nact_next;
      fc->nact_next = 0;
      fc->small_steps++;
      flip_next(fc);
    }
    cluster_barrier();
  }
#ifndef GQM_HOST_EMU
  if (graph && GQM_BLOCK0 && threadIdx.x == 0) cudaGraphSetConditional(h, fc->cond);
#endif
  (void)h;
  (void)graph;
  if (timed) ktimer_end(tm, start, items, wins);
}

}  // namespace gqm

// Whether a cluster of `csize` blocks of the small-step kernel can be resident
// on the current device (csize 8 or 16).  16 is beyond the portable cluster
// size and is allowed explicitly.
int gqm_flip_cluster_ok(int csize) {
#ifdef GQM_HOST_EMU
  return csize == 8 || csize == 16;
#else
  if (csize != 8 && csize != 16) return 0;
  int n0 = 0, n1 = 0;
  for (int pred = 0; pred < 2; ++pred) {
    const void *fn = pred ? (const void *)gqm::k_flip_small_cl<1> : (const void *)gqm::k_flip_small_cl<0>;
    if (csize > 8 && cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
      cudaGetLastError();
      return 0;
    }
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)csize;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3((unsigned)csize);
    cfg.blockDim = dim3(gqm::kClusterThreads);
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, fn, &cfg) != cudaSuccess) {
      cudaGetLastError();
      return 0;
    }
    (pred ? n1 : n0) = clusters;
  }
  return n0 > 0 && n1 > 0;
#endif
}

// Launch of k_flip_small_cl on the single-domain engine's buffers (refine.cu):
// one cluster of `csize` blocks.  mesh points at the caller's Mesh (the same
// layout in every compilation).
int gqm_flip_small_cl_launch(const void *mesh, size_t mesh_bytes, void *fc, int pred, int *act, uint8_t *clr,
                             int *win, int *ll, int *sl, int *fq, int *tl, int limit, int csize, cudaStream_t st,
                             cudaGraphConditionalHandle h, int graph, void *timer) {
  if (mesh_bytes != sizeof(gqm::Mesh) || (csize != 8 && csize != 16)) return GQM_ERR_ARGUMENT;
  gqm::Mesh M;
  memcpy(&M, mesh, sizeof(M));
  gqm::FlipCtl *c = static_cast<gqm::FlipCtl *>(fc);
  gqm::KTimer *tm = static_cast<gqm::KTimer *>(timer);
#ifdef GQM_HOST_EMU
  (void)st;
  if (pred)
    gqm::k_flip_small_cl<1>(M, c, act, clr, win, ll, sl, fq, tl, limit, h, graph, tm);
  else
    gqm::k_flip_small_cl<0>(M, c, act, clr, win, ll, sl, fq, tl, limit, h, graph, tm);
  return GQM_OK;
#else
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = (unsigned)csize;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3((unsigned)csize);
  cfg.blockDim = dim3(gqm::kClusterThreads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaError_t e = pred ? cudaLaunchKernelEx(&cfg, gqm::k_flip_small_cl<1>, M, c, act, clr, win, ll, sl, fq, tl,
                                            limit, h, graph, tm)
                       : cudaLaunchKernelEx(&cfg, gqm::k_flip_small_cl<0>, M, c, act, clr, win, ll, sl, fq, tl,
                                            limit, h, graph, tm);
  return e == cudaSuccess ? GQM_OK : GQM_ERR_CUDA;
#endif
}

// The incircle expansion-fallback counter of this translation unit's kernels
// (a device variable exists once per translation unit): added to *sum, then
// zeroed when `reset` is set.  Called by the single-domain driver, which
// reports the counters of all its kernels together.
int gqm_fallbacks_cluster(unsigned long long *sum, int reset, cudaStream_t st) {
  unsigned long long v = 0;
#ifdef GQM_HOST_EMU
  (void)st;
  v = gqm::g_incircle_fallbacks;
  if (reset) gqm::g_incircle_fallbacks = 0;
#else
  if (cudaMemcpyFromSymbolAsync(&v, gqm::g_incircle_fallbacks, sizeof(v), 0, cudaMemcpyDeviceToHost, st) !=
          cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return GQM_ERR_CUDA;
  if (reset) {
    const unsigned long long zero = 0;
    if (cudaMemcpyToSymbolAsync(gqm::g_incircle_fallbacks, &zero, sizeof(zero), 0, cudaMemcpyHostToDevice, st) !=
        cudaSuccess)
      return GQM_ERR_CUDA;
  }
#endif
  if (sum) *sum += v;
  return GQM_OK;
}
