// Host driver of the B200 refiner and the C ABI of include/gqm_refine.h.
//
// The driver reproduces the control flow of GPU_Refine_Quality
// (GPU_Refine/refine.cu:6500-7139): split encroached subsegments, then rounds
// of {mark bad triangles, split them, split encroached subsegments} until no
// bad triangle remains, then compact.  The reference's host bookkeeping of
// free slots (refine.cu:149-197, 3408-3444, 3545-3562, 5259-5296, 5354-5368)
// is reproduced exactly, because the slot a new point or triangle receives
// decides later conflicts.  Physical device buffers are allocated once, larger
// than the reference's logical capacity, and the logical capacity is tracked
// separately.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <atomic>
#include <initializer_list>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/gqm_refine.h"
#include "host_copy.h"
#include "kernels.cuh"

// NVTX ranges around the driver's phases (refinement, encroached-subsegment
// splitting, Steiner rounds, flip-flop loops, output compaction, result
// download) for a profiler's timeline; with no profiler attached a range
// costs a few nanoseconds.
#ifndef GQM_HOST_EMU
#include <nvtx3/nvToolsExt.h>
struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange &) = delete;
  NvtxRange &operator=(const NvtxRange &) = delete;
};
#else
struct NvtxRange {
  explicit NvtxRange(const char *) {}
};
#endif

// batch.cu: the flip steps of small active sets in one block
int gqm_flip_small_launch(const void *mesh, size_t mesh_bytes, void *fc, int pred, int *act, uint8_t *clr, int *win,
                          int *ll, int *sl, int *fq, int *tl, int limit, cudaStream_t st,
                          cudaGraphConditionalHandle h, int graph, void *timer);
// flipcl.cu: the same on one thread-block cluster of csize blocks
int gqm_flip_small_cl_launch(const void *mesh, size_t mesh_bytes, void *fc, int pred, int *act, uint8_t *clr,
                             int *win, int *ll, int *sl, int *fq, int *tl, int limit, int csize, cudaStream_t st,
                             cudaGraphConditionalHandle h, int graph, void *timer);
int gqm_flip_cluster_ok(int csize);
// the incircle expansion-fallback counters of batch.cu's and flipcl.cu's kernels
int gqm_fallbacks_cta(unsigned long long *sum, int reset, cudaStream_t st);
int gqm_fallbacks_cluster(unsigned long long *sum, int reset, cudaStream_t st);

namespace gqm {

// ============================================================================
// Ordered stream compaction: out[k] = map(i) for the k-th i in [lo, hi) with
// pred(i), in ascending i.  Three launches: per-block counts, one-block scan,
// per-block ordered emit (warp ballots).  No spin waits.
// ============================================================================
constexpr int kCompactThreads = 256;
constexpr int kCompactItems = 16;  // consecutive elements per thread
constexpr int kCompactTile = kCompactThreads * kCompactItems;
constexpr int kMaxCompactBlocks = 2048;

// per-block counts: block b covers [lo + b*chunk, lo + (b+1)*chunk)
template <class F>
__global__ void __launch_bounds__(kCompactThreads) k_cnt(F f, int lo, int hi, int chunk, int *bc) {
  int b0 = lo + blockIdx.x * chunk, b1 = min(hi, b0 + chunk);
  int c = 0;
  for (int s = b0 + threadIdx.x * kCompactItems; s < b1; s += kCompactTile) {
#pragma unroll
    for (int j = 0; j < kCompactItems; ++j)
      if (s + j < b1 && f(s + j)) ++c;
  }
  __shared__ int red[32];
  for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x < 32) {
    int v = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) bc[blockIdx.x] = v;
  }
}
// exclusive scan of bc[0..nb) in place (one block of 1024 threads); total at *total
__global__ void k_scan(int *bc, int nb, int *total) {
  __shared__ int sh[1024];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < nb; base += 1024) {
    int i = base + threadIdx.x;
    int v = (i < nb) ? bc[i] : 0;
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
      int t = (threadIdx.x >= o) ? sh[threadIdx.x - o] : 0;
      __syncthreads();
      sh[threadIdx.x] += t;
      __syncthreads();
    }
    if (i < nb) bc[i] = carry + sh[threadIdx.x] - v;
    __syncthreads();
    if (threadIdx.x == 1023) carry += sh[1023];
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}
// ordered emit: each thread takes 16 consecutive elements of a 4096-element
// tile, a block-wide exclusive scan of the per-thread counts gives the slots.
// With total set (a one-block compaction, bc pointing at a zero), the block
// also writes the count, so a range of one block needs no count or scan launch.
template <class F, class Mp>
__global__ void __launch_bounds__(kCompactThreads) k_emit(F f, Mp m, int lo, int hi, int chunk, const int *bc,
                                                          int *out, int *total) {
  __shared__ int wsum[kCompactThreads / 32];
  int b0 = lo + blockIdx.x * chunk, b1 = min(hi, b0 + chunk);
  int base = bc[blockIdx.x];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int tile = b0; tile < b1; tile += kCompactTile) {
    int s = tile + threadIdx.x * kCompactItems;
    unsigned bits = 0;
#pragma unroll
    for (int j = 0; j < kCompactItems; ++j)
      if (s + j < b1 && f(s + j)) bits |= 1u << j;
    int c = __popc(bits);
    // inclusive warp scan of c
    int x = c;
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    int woff = 0, tot = 0;
#pragma unroll
    for (int w = 0; w < kCompactThreads / 32; ++w) {
      int v = wsum[w];
      woff += (w < warp) ? v : 0;
      tot += v;
    }
    int pos = base + woff + x - c;
    while (bits) {
      int j = __ffs(bits) - 1;
      bits &= bits - 1;
      out[pos++] = m(s + j);
    }
    base += tot;
    __syncthreads();
  }
  if (total && threadIdx.x == 0) *total = base;
}

// predicates and maps for the compactions
struct Ident {
  __device__ int operator()(int i) const { return i; }
};
struct ValueOf {
  const int *a;
  __device__ int operator()(int i) const { return a[i]; }
};
struct PNotNullFlag {
  const uint8_t *tst, *flag;
  __device__ bool operator()(int i) const { return (tst[i] & TS_NOTNULL) && flag[i]; }
};
struct PWinner {
  const uint8_t *tst, *tfo;
  __device__ bool operator()(int i) const { return (tst[i] & TS_NOTNULL) && tfo[i] != 15; }
};
struct PNeg {
  const int *a;
  __device__ bool operator()(int i) const { return a[i] < 0; }
};
struct PNonNeg {
  const int *a;
  __device__ bool operator()(int i) const { return a[i] >= 0; }
};
struct PBad {
  const uint8_t *tst;
  __device__ bool operator()(int i) const { return (tst[i] & (TS_NOTNULL | TS_BAD)) == (TS_NOTNULL | TS_BAD); }
};
struct PTriNull {
  const uint8_t *tst;
  __device__ bool operator()(int i) const { return !(tst[i] & TS_NOTNULL); }
};
struct PTriLive {
  const uint8_t *tst;
  __device__ bool operator()(int i) const { return (tst[i] & TS_NOTNULL) != 0; }
};
struct PPtDeleted {
  const uint8_t *ps;
  __device__ bool operator()(int i) const { return (ps[i] & PS_DELETED) != 0; }
};
struct PPtLive {
  const uint8_t *ps;
  __device__ bool operator()(int i) const { return !(ps[i] & PS_DELETED); }
};

__global__ void k_fill(int *a, int n, int v) { GS_LOOP(i, n) a[i] = v; }
__global__ void k_copy(int *dst, const int *src, const int *dn) {
  int n = *dn;
  GS_LOOP(i, n) dst[i] = src[i];
}
__global__ void k_set_count(int *dst, int v) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *dst = v;
}

// ============================================================================
// Refiner
// ============================================================================
struct Refiner {
  cudaStream_t st = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int device = 0;
  Mesh M{};
  // physical capacities
  long pphys = 0, tphys = 0, sphys = 0;
  // reference logical state
  long pcap = 0, tcap = 0;
  int last_point = 0, last_triangle = 0, last_subseg = 0, nseg_in = 0;
  int pointblock = 0, triblock = 0, nempty_p = 0, nempty_t = 0, lenp = 0, lent = 0;
  // per-triangle scratch (capacity tphys)
  int *emptyt = nullptr, *bad = nullptr, *imark = nullptr, *ilist = nullptr, *sinks = nullptr, *wl = nullptr;
  int *act = nullptr, *win = nullptr, *neg = nullptr, *ll = nullptr, *sl = nullptr, *newidx = nullptr;
  int *tail = nullptr;
  double2 *center = nullptr;
  int *cav = nullptr, *cavn = nullptr;  // stored cavities of the Steiner candidates
  long cav_cap = 0;
  int *fq = nullptr, *tl = nullptr;  // flip-step queue and claimed-triangle list
  uint8_t *clr = nullptr;            // deferred flag clears of a flip step
  FlipCtl *fc = nullptr;             // flip-loop control block (device)
  KTimer *ktm = nullptr;             // launch timer of the flip-step check kernel
  KTimer *stm = nullptr;             // launch timer of the small-step kernel
  bool probing = false;              // events around every flip-loop launch
  std::vector<cudaEvent_t> loop_ev;  // pairs, reused every run
  size_t loop_ev_used = 0;
  double probe_loop_ms = 0.0;
  long long probe_loops = 0;
  // the flip-flop loop as a CUDA graph with a device-side while condition
  bool use_graph = true;
  cudaGraph_t flip_graph = nullptr;
  cudaGraphExec_t flip_exec = nullptr;
  Mesh flip_graph_mesh{};
  int flip_graph_pred = -1;
  // per-point scratch (capacity pphys)
  int *emptyp = nullptr, *pnew = nullptr;
  // per-subsegment scratch (capacity sphys)
  int *enclist = nullptr, *encl2 = nullptr, *smark = nullptr, *mids = nullptr, *snap = nullptr;
  int2 *segs = nullptr;
  // counters and small buffers
  int *dcount = nullptr;  // [16] list sizes on the device
  int *hcount = nullptr;  // pinned mirror
  int *bc = nullptr;      // compaction block counts
  unsigned long long *dctr = nullptr;  // [8] event counters (Steiner, midpoints, -, -, learned candidates, used)
  double *dgc = nullptr;
  int *dinput = nullptr;  // staging for host inputs
  size_t dinput_bytes = 0;
  // kept between runs (grow only): pinned host staging of inputs and results,
  // the device result block, segment copy and the initSubsegs hash
  char *h_stage = nullptr, *d_out = nullptr;
  size_t h_stage_cap = 0, d_out_cap = 0, segs_cap = 0, hash_cap = 0;
  unsigned long long *hkeys = nullptr;
  int *hvals = nullptr, *s2ti = nullptr;
  // options
  int pred_mode = 0, mode = 1, offcenter = 1, offconstant = 0;
  // learned Steiner placement: the network on the device
  int placement = GQM_PLACE_PLAIN;
  uint16_t *mlp_w = nullptr;
  float *mlp_b = nullptr;
  // training-data collection (gqm_learn_collect): device rows and their count
  float *col_feat = nullptr, *col_tgt = nullptr;
  unsigned long long *col_cnt = nullptr, col_cap = 0;
  double theta = 20.0;
  long long max_rounds = 1000000;
  gqm_stats stats{};
  int status = 0;
  // result sizes
  int out_np = 0, out_nt = 0, out_ns = 0;
  bool have_result = false;
  long long flip_prof_steps[kFlipProfileBins] = {}, flip_prof_items[kFlipProfileBins] = {};

  enum { C_LIST0 = 0, C_LIST1, C_LIST2, C_LIST3, C_LIST4, C_LIST5, C_MISC, C_QN, C_TN };

  ~Refiner() { release(); }

  template <class T>
  static cudaError_t dalloc(T **p, size_t n) {
    *p = nullptr;
    return cudaMalloc((void **)p, sizeof(T) * std::max<size_t>(n, 1));
  }
  // grow-only buffers kept between runs
  int grow_pinned(size_t need) {
    if (need <= h_stage_cap) return GQM_OK;
    if (h_stage) cudaFreeHost(h_stage);
    h_stage = nullptr;
    h_stage_cap = 0;
    if (cudaMallocHost((void **)&h_stage, need) != cudaSuccess) {
      h_stage = nullptr;
      return GQM_ERR_MEMORY;
    }
    h_stage_cap = need;
    return GQM_OK;
  }
  template <class T>
  int grow_dev(T **q, size_t *cap, size_t n) {
    if (n <= *cap && *q) return GQM_OK;
    if (*q) cudaFree(*q);
    *cap = 0;
    if (dalloc(q, n) != cudaSuccess) {
      *q = nullptr;
      return GQM_ERR_MEMORY;
    }
    *cap = n;
    return GQM_OK;
  }
  // grow a device array to n elements, keeping its first `keep` elements
  template <class T>
  cudaError_t regrow(T **p, size_t keep, size_t n) {
    T *q = nullptr;
    cudaError_t e = dalloc(&q, n);
    if (e != cudaSuccess) return e;
    if (*p && keep) cudaMemcpyAsync(q, *p, sizeof(T) * keep, cudaMemcpyDeviceToDevice, st);
    if (*p) {
      cudaStreamSynchronize(st);
      cudaFree(*p);
    }
    *p = q;
    return cudaSuccess;
  }

  void drop_flip_graph() {
#ifndef GQM_HOST_EMU
    if (flip_exec) cudaGraphExecDestroy(flip_exec);
    if (flip_graph) cudaGraphDestroy(flip_graph);
#endif
    flip_exec = nullptr;
    flip_graph = nullptr;
  }

  void release() {
    drop_flip_graph();
    void *ptrs[] = {M.pts, M.ps, M.pred, M.tv, M.tn, M.tsg, M.tst, M.tflip, M.tfo, M.flip0, M.tmark, M.tpos,
                    M.s2t, M.s2seg, M.enc, M.err, stm, emptyt, bad, imark, ilist, sinks, wl, act, win, neg, ll, sl,
                    newidx, tail, center, emptyp, pnew, enclist, encl2, smark, mids, snap, segs, dcount, bc,
                    dctr, dgc, dinput, mlp_w, mlp_b, M.fstamp, M.tstamp, fq, tl, clr, fc, cav, cavn, ktm, M.wbits, M.wcnt, M.wsup, M.wmeg};
    for (void *p : ptrs)
      if (p) cudaFree(p);
    if (hcount) cudaFreeHost(hcount);
    hcount = nullptr;
    M = Mesh{};
    emptyt = bad = imark = ilist = sinks = wl = act = win = neg = ll = sl = newidx = tail = nullptr;
    fq = tl = nullptr;
    clr = nullptr;
    fc = nullptr;
    ktm = nullptr;
    stm = nullptr;
    mlp_w = nullptr;
    mlp_b = nullptr;
    for (cudaEvent_t e : loop_ev) cudaEventDestroy(e);
    loop_ev.clear();
    loop_ev_used = 0;
    center = nullptr;
    cav = cavn = nullptr;
    cav_cap = 0;
    emptyp = pnew = enclist = encl2 = smark = mids = snap = nullptr;
    segs = nullptr;
    dcount = bc = nullptr;
    dctr = nullptr;
    dgc = nullptr;
    dinput = nullptr;
    dinput_bytes = 0;
    if (h_stage) cudaFreeHost(h_stage);
    for (void *q : {(void *)d_out, (void *)hkeys, (void *)hvals, (void *)s2ti})
      if (q) cudaFree(q);
    h_stage = d_out = nullptr;
    hkeys = nullptr;
    hvals = s2ti = nullptr;
    h_stage_cap = d_out_cap = segs_cap = hash_cap = 0;
    pphys = tphys = sphys = 0;
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    ev0 = ev1 = nullptr;
    if (st) cudaStreamDestroy(st);
    st = nullptr;
  }

  int setup(int dev) {
    device = dev;
    if (cudaSetDevice(dev) != cudaSuccess) return GQM_ERR_NO_DEVICE;
    if (!st && cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return GQM_ERR_CUDA;
    if (!ev0) cudaEventCreate(&ev0);
    if (!ev1) cudaEventCreate(&ev1);
    if (!dcount) {
      if (dalloc(&dcount, 16) || dalloc(&bc, kMaxCompactBlocks + 1) || dalloc(&dctr, 8) || dalloc(&dgc, 2) ||
          dalloc(&M.err, 1) || dalloc(&fc, 1) || dalloc(&ktm, 1) || dalloc(&stm, 1))
        return GQM_ERR_MEMORY;
      cudaMemsetAsync(fc, 0, sizeof(FlipCtl), st);
      cudaMemsetAsync(ktm, 0, sizeof(KTimer), st);  // off until gqm_context_probe
      cudaMemsetAsync(stm, 0, sizeof(KTimer), st);
      cudaMemsetAsync(bc + kMaxCompactBlocks, 0, sizeof(int), st);  // the zero base of one-block compactions
#ifdef GQM_HOST_EMU
      use_graph = false;
#else
      const char *ng = getenv("GQM_NO_GRAPH");
      use_graph = !(ng && ng[0] == '1');
#endif
      if (cudaMallocHost((void **)&hcount, sizeof(int) * 16) != cudaSuccess) return GQM_ERR_MEMORY;
    }
    return GQM_OK;
  }

  static int grid_for(long n, int threads = 256) {
    long g = (n + threads - 1) / threads;
    if (g < 1) g = 1;
    if (g > 148L * 64) g = 148L * 64;
    return (int)g;
  }
#ifdef GQM_HOST_EMU
#define KL(kernel, g, b) kernel
#else
#define KL(kernel, g, b) kernel<<<(g), (b), 0, st>>>
#endif
#define LAUNCH(kernel, n, ...)                   \
  do {                                           \
    KL(kernel, grid_for(n), 256)(__VA_ARGS__);   \
    stats.kernel_launches++;                     \
  } while (0)

  // Ordered compaction over [lo, hi) into out; the count lands in dcount[slot].
  template <class F, class Mp>
  void compact(F f, Mp m, int lo, int hi, int *out, int slot) {
    compact_to(f, m, lo, hi, out, dcount + slot);
  }
  template <class F, class Mp>
  void compact_to(F f, Mp m, int lo, int hi, int *out, int *dcnt) {
    int n = hi - lo;
#ifdef GQM_HOST_EMU
    int c = 0;
    for (int i = lo; i < hi; ++i)
      if (f(i)) out[c++] = m(i);
    *dcnt = c;
    stats.kernel_launches += 3;
    return;
#endif
    if (n <= 0) {
      KL(k_set_count, 1, 32)(dcnt, 0);
      stats.kernel_launches++;
      return;
    }
    int chunk = std::max(kCompactTile, (n + kMaxCompactBlocks - 1) / kMaxCompactBlocks);
    chunk = (chunk + kCompactTile - 1) / kCompactTile * kCompactTile;
    int nb = (n + chunk - 1) / chunk;
    if (nb == 1) {  // one block: emit and count in one launch (bc[kMaxCompactBlocks] stays 0)
      KL(k_emit, 1, kCompactThreads)(f, m, lo, hi, chunk, bc + kMaxCompactBlocks, out, dcnt);
      stats.kernel_launches++;
      return;
    }
    KL(k_cnt, nb, kCompactThreads)(f, lo, hi, chunk, bc);
    KL(k_scan, 1, 1024)(bc, nb, dcnt);
    KL(k_emit, nb, kCompactThreads)(f, m, lo, hi, chunk, bc, out, nullptr);
    stats.kernel_launches += 3;
  }
  int fetch(int slot) {
    cudaMemcpyAsync(hcount + slot, dcount + slot, sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    stats.host_syncs++;
    return hcount[slot];
  }
  int check_device_error() {
    int e = 0;
    cudaMemcpyAsync(hcount + C_MISC, M.err, sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaError_t ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess) return GQM_ERR_CUDA;
    e = hcount[C_MISC];
    return e;
  }

  // ---- capacity management ----
  int alloc_points(long n) {
    long old = pphys;
    if (n <= old) return GQM_OK;
    if (regrow(&M.pts, old, n) || regrow(&M.ps, old, n) || regrow(&M.pred, old, n) || regrow(&emptyp, 0, n) ||
        regrow(&pnew, old, n) || regrow(&tail, 0, std::max<long>(n, tphys)))
      return GQM_ERR_MEMORY;
    // new slots are deleted points
    if (n > old) {
      cudaMemsetAsync(M.ps + old, PS_DELETED, n - old, st);
      cudaMemsetAsync(M.pred + old, 0, n - old, st);
      cudaMemsetAsync(M.pts + old, 0, sizeof(double2) * (n - old), st);
    }
    pphys = n;
    return GQM_OK;
  }
  int alloc_tris(long n) {
    long old = tphys;
    if (n <= old) return GQM_OK;
    if (regrow(&M.tv, old, n) || regrow(&M.tn, old, n) || regrow(&M.tsg, old, n) || regrow(&M.tst, old, n) ||
        regrow(&M.tflip, old, n) || regrow(&M.tfo, old, n) || regrow(&M.flip0, old, n) ||
        regrow(&M.tmark, old, n) || regrow(&M.tpos, old, n) || regrow(&emptyt, 0, n) || regrow(&bad, old, n) ||
        regrow(&imark, old, n) || regrow(&ilist, old, n) || regrow(&sinks, old, n) || regrow(&wl, old, n) ||
        regrow(&act, old, n) || regrow(&win, old, n) || regrow(&neg, old, n) || regrow(&ll, 2 * old, 2 * n) ||
        regrow(&sl, 6 * old, 6 * n) || regrow(&newidx, 0, n) || regrow(&tail, 0, std::max<long>(n, pphys)) ||
        regrow(&center, old, n) || regrow(&M.fstamp, old, n) || regrow(&M.tstamp, old, n) || regrow(&fq, 0, n) ||
        regrow(&tl, 0, n) || regrow(&clr, 0, n) || regrow(&M.wbits, 0, n / 32 + 1) ||
        regrow(&M.wcnt, 0, n / 1024 + 1) || regrow(&M.wsup, 0, n / 32768 + 1) ||
        regrow(&M.wmeg, 0, n / 1048576 + 1))
      return GQM_ERR_MEMORY;
    // winner bitmap and chunk counts are all zero between flip steps
    cudaMemsetAsync(M.wbits, 0, sizeof(unsigned) * (n / 32 + 1), st);
    cudaMemsetAsync(M.wcnt, 0, sizeof(int) * (n / 1024 + 1), st);
    cudaMemsetAsync(M.wsup, 0, sizeof(int) * (n / 32768 + 1), st);
    cudaMemsetAsync(M.wmeg, 0, sizeof(int) * (n / 1048576 + 1), st);
    if (n > old) {
      cudaMemsetAsync(M.tst + old, 0, n - old, st);
      cudaMemsetAsync(M.tflip + old, 0, n - old, st);
      cudaMemsetAsync(M.tfo + old, 0, n - old, st);
      cudaMemsetAsync(M.tsg + old, 0xff, sizeof(int4) * (n - old), st);
      cudaMemsetAsync(M.tpos + old, 0xff, sizeof(int) * (n - old), st);
      cudaMemsetAsync(M.fstamp + old, 0, sizeof(int) * (n - old), st);
      cudaMemsetAsync(M.tstamp + old, 0, sizeof(int) * (n - old), st);
    }
    tphys = n;
    return GQM_OK;
  }
  int alloc_subsegs(long n) {
    long old = sphys;
    if (n <= old) return GQM_OK;
    if (regrow(&M.s2t, old, n) || regrow(&M.s2seg, old, n) || regrow(&M.enc, old, n) || regrow(&enclist, old, n) ||
        regrow(&encl2, old, n) || regrow(&smark, old, n) || regrow(&mids, old, n) || regrow(&snap, old, n))
      return GQM_ERR_MEMORY;
    // new subsegment entries start at epoch 0 so that the first tagged store wins
    cudaMemsetAsync(M.s2t + old, 0, sizeof(s2t_t) * (n - old), st);
    sphys = n;
    return GQM_OK;
  }

  // updateEmptyPoints / updateEmptyTriangles (refine.cu:149-197)
  int refresh_points() {
    compact(PPtDeleted{M.ps}, Ident{}, 0, (int)pcap, emptyp, C_MISC);
    lenp = fetch(C_MISC);
    return lenp;
  }
  int refresh_tris() {
    compact(PTriNull{M.tst}, Ident{}, 0, (int)tcap, emptyt, C_MISC);
    lent = fetch(C_MISC);
    return lent;
  }
  // growth steps of refine.cu:3408-3444 / 5259-5296
  int ensure_slots(int npts, int ntris) {
    if (npts > nempty_p) {
      nempty_p = refresh_points();
      long num = 0;
      while (npts > nempty_p + num * pointblock) num++;
      if (num) {
        long ncap = pcap + num * pointblock;
        if (ncap > pphys) {
#ifdef GQM_TEST_TIGHT_BUFFERS
          int rc = alloc_points(ncap);
#else
          int rc = alloc_points(std::max(ncap, pphys + pphys / 2));
#endif
          if (rc) return rc;
        }
        pcap = ncap;
        nempty_p = refresh_points();
      }
    }
    if (ntris > nempty_t) {
      nempty_t = refresh_tris();
      long num = 0;
      while (ntris > nempty_t + num * triblock) num++;
      if (num) {
        long ncap = tcap + num * triblock;
        if (ncap > tphys) {
#ifdef GQM_TEST_TIGHT_BUFFERS
          int rc = alloc_tris(ncap);
#else
          int rc = alloc_tris(std::max(ncap, tphys + tphys / 2));
#endif
          if (rc) return rc;
        }
        tcap = ncap;
        nempty_t = refresh_tris();
      }
    }
    return GQM_OK;
  }
  // slot bookkeeping after an insertion batch (refine.cu:3545-3559, 5354-5368)
  void consume_slots(int npts, int ntris) {
    int slot_after = (int)(pcap - last_point);
    int slot_before = nempty_p - slot_after;
    if (slot_before < npts) last_point += npts - slot_before;
    nempty_p -= npts;
    slot_after = (int)(tcap - last_triangle);
    slot_before = nempty_t - slot_after;
    if (slot_before < ntris) last_triangle += ntris - slot_before;
    nempty_t -= ntris;
  }
  const int *pslots() const { return emptyp + (lenp - nempty_p); }
  const int *tslots() const { return emptyt + (lent - nempty_t); }

  // ---- flip-flop (refine.cu:2328-2490), driven by active sets ----
  // One step: check (A) -> winners (W) -> link+phase 1 -> phase 2 -> phase 3
  // -> redundant points -> reset claims -> next A -> loop condition.  Every
  // count lives in the control block, so the whole loop runs on the device.
#ifndef GQM_STEP_GRID
#define GQM_STEP_GRID (148 * 4)
#endif
  // steps whose active set has at most this many triangles run in one launch
#ifndef GQM_SMALL_STEP
#define GQM_SMALL_STEP 1024
#endif
  // Launch shape of the flip-flop loop (gqm_tuning).  None of it changes a
  // result: every step makes the reference's decisions whatever the grid.
  struct Tuning {
    int step_grid = GQM_STEP_GRID;       // blocks of each grid-wide step kernel
    int small_limit = GQM_SMALL_STEP;    // <= this many active triangles: small-step kernel (0: never)
    int small_cluster = 1;               // small-step kernel: 1 = one 512-thread block, 8 / 16 = a cluster
    int check_minb = GQM_WALK_MIN_BLOCKS;  // register budget of the check kernel (blocks per SM)
    bool operator==(const Tuning &o) const {
      return step_grid == o.step_grid && small_limit == o.small_limit && small_cluster == o.small_cluster &&
             check_minb == o.check_minb;
    }
  } tune, flip_graph_tune;
  template <int PRED>
  void launch_check(const TouchL &T) {
    void (*check)(Mesh, const int *, const int *, uint8_t *, TouchL, KTimer *) =
        tune.check_minb == 1 ? k_check_flip2<PRED, 1> : k_check_flip2<PRED, 2>;
    KL(check, tune.step_grid, 256)(M, act, &fc->nact, clr, T, ktm);
  }
  void flip_body(cudaGraphConditionalHandle h, int graph) {
    FlipQ Q{fq, &fc->qn, &fc->gen};
    TouchL T{tl, &fc->tn, &fc->gen};
    const int g = tune.step_grid;
    if (pred_mode)
      launch_check<1>(T);
    else
      launch_check<0>(T);
    KL(k_flip_winner2, g, 256)(M, act, &fc->nact, clr, Q, win, &fc->winn);
    KL(k_link_phase1, g, 256)(M, win, &fc->winn, ll, sl, &fc->epoch);
    KL(k_phase2, g, 256)(M, win, &fc->winn, ll, sl);
    KL(k_phase3q, g, 256)(M, win, &fc->winn, sl, Q);
    KL(k_mark_red_steiner_q, g, 256)(M, tl, &fc->tn, Q);
    KL(k_flip_reset_filter, g, 256)(M, tl, &fc->tn, fq, &fc->qn, act, &fc->nact_next);
    KL(k_flip_cond, 1, 32)(fc, h, graph);
    // the following small steps in one block (batch.cu) or one cluster
    // (flipcl.cu), which re-sets the condition
    if (tune.small_limit <= 0) return;
    if (tune.small_cluster > 1)
      gqm_flip_small_cl_launch(&M, sizeof(M), fc, pred_mode, act, clr, win, ll, sl, fq, tl, tune.small_limit,
                               tune.small_cluster, st, h, graph, stm);
    else
      gqm_flip_small_launch(&M, sizeof(M), fc, pred_mode, act, clr, win, ll, sl, fq, tl, tune.small_limit, st, h,
                            graph, stm);
  }
  // kernels one grid step of the loop body launches (with its condition kernel)
  int step_kernels() const { return tune.small_limit > 0 ? 9 : 8; }
  int build_flip_graph() {
#ifdef GQM_HOST_EMU
    return GQM_ERR_CUDA;
#else
    drop_flip_graph();
    cudaGraph_t g = nullptr;
    if (cudaGraphCreate(&g, 0) != cudaSuccess) return GQM_ERR_CUDA;
    cudaGraphConditionalHandle h;
    if (cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault) != cudaSuccess) {
      cudaGraphDestroy(g);
      return GQM_ERR_CUDA;
    }
    // node 1: k_flip_prep sets the condition for the first step
    if (cudaStreamBeginCaptureToGraph(st, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      cudaGraphDestroy(g);
      return GQM_ERR_CUDA;
    }
    k_flip_prep<<<1, 32, 0, st>>>(fc, h, 1);
    cudaGraph_t gc = nullptr;
    if (cudaStreamEndCapture(st, &gc) != cudaSuccess) {
      cudaGraphDestroy(g);
      return GQM_ERR_CUDA;
    }
    cudaGraphNode_t prep = nullptr;
    size_t nn = 1;
    if (cudaGraphGetNodes(g, &prep, &nn) != cudaSuccess || nn != 1) {
      cudaGraphDestroy(g);
      return GQM_ERR_CUDA;
    }
    // node 2: while (condition) { step }
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t cn = nullptr;
    if (cudaGraphAddNode(&cn, g, &prep, 1, &cp) != cudaSuccess) {
      cudaGraphDestroy(g);
      return GQM_ERR_CUDA;
    }
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    if (cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) !=
        cudaSuccess) {
      cudaGraphDestroy(g);
      return GQM_ERR_CUDA;
    }
    flip_body(h, 1);
    cudaGraph_t bc2 = nullptr;
    if (cudaStreamEndCapture(st, &bc2) != cudaSuccess) {
      cudaGraphDestroy(g);
      return GQM_ERR_CUDA;
    }
    if (cudaGraphInstantiate(&flip_exec, g, 0) != cudaSuccess) {
      cudaGraphDestroy(g);
      flip_exec = nullptr;
      return GQM_ERR_CUDA;
    }
    flip_graph = g;
    flip_graph_mesh = M;
    flip_graph_pred = pred_mode;
    flip_graph_tune = tune;
    return GQM_OK;
#endif
  }
  // next pair of probe events (nullptr when none can be created)
  cudaEvent_t *loop_events() {
    while (loop_ev.size() < 2 * (loop_ev_used + 1)) {
      cudaEvent_t e;
      if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
      loop_ev.push_back(e);
    }
    return &loop_ev[2 * loop_ev_used++];
  }
  // after the run's final sync: add the probe events' intervals to the totals
  void collect_loop_events() {
    for (size_t i = 0; i < loop_ev_used; ++i) {
      float ms = 0.0f;
      if (cudaEventElapsedTime(&ms, loop_ev[2 * i], loop_ev[2 * i + 1]) == cudaSuccess) probe_loop_ms += ms;
      probe_loops++;
    }
    loop_ev_used = 0;
  }
  int flip_flop(int ntri) {
    NvtxRange nvtx("gqm:flip_flop");
    LAUNCH(k_flip_entry_reset, ntri, M, ntri);
    compact_to(PNotNullFlag{M.tst, M.tflip}, Ident{}, 0, ntri, act, &fc->nact);
    if (use_graph) {
      if (!flip_exec || memcmp(&flip_graph_mesh, &M, sizeof(Mesh)) != 0 || flip_graph_pred != pred_mode ||
          !(flip_graph_tune == tune)) {
        if (build_flip_graph() != GQM_OK) {
          use_graph = false;
          cudaGetLastError();
        }
      }
    }
    if (use_graph) {
      cudaEvent_t *ev = probing ? loop_events() : nullptr;
      if (ev) cudaEventRecord(ev[0], st);
      if (cudaGraphLaunch(flip_exec, st) != cudaSuccess) return GQM_ERR_CUDA;
      if (ev) cudaEventRecord(ev[1], st);
      stats.kernel_launches++;
      return GQM_OK;
    }
    cudaGraphConditionalHandle h{};
    KL(k_flip_prep, 1, 32)(fc, h, 0);
    stats.kernel_launches++;
    for (;;) {
      cudaMemcpyAsync(hcount + C_MISC, &fc->cond, sizeof(int), cudaMemcpyDeviceToHost, st);
      cudaStreamSynchronize(st);
      stats.host_syncs++;
      if (!hcount[C_MISC]) break;
      flip_body(h, 0);
      stats.kernel_launches += step_kernels();
    }
    return GQM_OK;
  }

  // ---- splitEncsegs (refine.cu:3180-3778) ----
  int split_encsegs() {
    NvtxRange nvtx("gqm:split_encsegs");
    long long outer = 0;
    for (;;) {
      compact(PNonNeg{M.enc}, Ident{}, 0, last_subseg, enclist, C_LIST0);
      int nenc = fetch(C_LIST0);
      if (nenc == 0) break;
      if (++outer > max_rounds) return GQM_ERR_ROUND_LIMIT;
      // delete free Steiner points inside diametral circles
      LAUNCH(k_copy, nenc, smark, enclist, dcount + C_LIST0);
      int nmark = nenc;
      long long inner = 0;
      for (;;) {
        compact(PNonNeg{smark}, ValueOf{smark}, 0, nmark, mids, C_LIST1);
        int ndel = fetch(C_LIST1);
        if (ndel == 0) break;
        if (++inner > max_rounds) return GQM_ERR_ROUND_LIMIT;
        nmark = ndel;
        LAUNCH(k_mark_redundant, ndel, M, smark, mids, dcount + C_LIST1);
        int rc = flip_flop(last_triangle);
        if (rc) return rc;
      }
      int rc = ensure_slots(nenc, 2 * nenc);
      if (rc) return rc;
      if (last_subseg + nenc > sphys) {
        rc = alloc_subsegs(std::max<long>(last_subseg + nenc, sphys + sphys / 2));
        if (rc) return rc;
      }
      LAUNCH(k_fill, nenc, M.enc + last_subseg, nenc, -1);
      LAUNCH(k_copy, nenc, smark, enclist, dcount + C_LIST0);
      long long mid_iter = 0;
      for (;;) {
        compact(PNonNeg{smark}, Ident{}, 0, nenc, mids, C_LIST1);
        int nmid = fetch(C_LIST1);
        if (nmid == 0) break;
        if (++mid_iter > 64 * max_rounds) return GQM_ERR_ROUND_LIMIT;
        LAUNCH(k_reset_mid, nmid, M, mids, dcount + C_LIST1, smark);
        LAUNCH(k_mark_mid, nmid, M, mids, dcount + C_LIST1, smark);
        LAUNCH(k_mid_snapshot, nmid, M, mids, dcount + C_LIST1, smark, snap);
        KL(k_bump_epoch, 1, 32)(fc);
        LAUNCH(k_insert_mid, nmid, M, mids, dcount + C_LIST1, smark, snap, pslots(), tslots(), last_subseg,
               &fc->epoch, dctr + 1);
        LAUNCH(k_update_mid_nbrs, nmid, M, mids, dcount + C_LIST1, smark, enclist);
      }
      consume_slots(nenc, 2 * nenc);
      last_subseg += nenc;
      rc = flip_flop(last_triangle);
      if (rc) return rc;
    }
    return GQM_OK;
  }

  // ---- splitTriangles (refine.cu:5107-5547) ----
  int split_triangles(int nbad) {
    NvtxRange nvtx("gqm:split_triangles");
    int *dn = dcount + C_LIST2;  // number of bad triangles
    LAUNCH(k_copy, nbad, imark, bad, dn);
    LAUNCH(k_copy, nbad, ilist, bad, dn);
    LAUNCH(k_circumcenter, nbad, M, bad, dn, (double)offconstant, offcenter, center);
    if (col_feat) LAUNCH(k_collect, nbad, M, bad, dn, center, col_feat, col_tgt, col_cnt, col_cap);
    if (placement == GQM_PLACE_LEARNED) {  // two warps of a block take 64 candidates per pass
      KL(k_learned_place, std::max(1, std::min((nbad + 63) / 64, 148 * 8)), 64)(M, bad, dn, mlp_dev(mlp_w, mlp_b),
                                                                                center, dctr + 4);
      stats.kernel_launches++;
    }
    LAUNCH(k_fill, last_triangle, M.tmark, last_triangle, kMaxInt);
    if (pred_mode)
      LAUNCH(k_locate<1>, nbad, M, bad, dn, center, sinks);
    else
      LAUNCH(k_locate<0>, nbad, M, bad, dn, center, sinks);
    LAUNCH(k_remove_losers, nbad, M, bad, dn, sinks, imark);
    LAUNCH(k_fill, last_triangle, M.tmark, last_triangle, kMaxInt);
    if (nbad > cav_cap) {  // stored cavities: kCavityCap rows of nbad entries
      long cap = std::max<long>(nbad, 2 * cav_cap);
      cudaStreamSynchronize(st);
      if (cav) cudaFree(cav);
      if (cavn) cudaFree(cavn);
      cav = cavn = nullptr;
      cav_cap = 0;
      if (dalloc(&cav, (size_t)kCavityCap * cap) || dalloc(&cavn, cap)) return GQM_ERR_MEMORY;
      cav_cap = cap;
    }
    if (pred_mode)
      LAUNCH(k_cavity_mark<1>, nbad, M, dn, sinks, center, imark, ilist, cav, cavn, nbad);
    else
      LAUNCH(k_cavity_mark<0>, nbad, M, dn, sinks, center, imark, ilist, cav, cavn, nbad);
    LAUNCH(k_cavity_check, nbad, M, dn, cav, cavn, nbad, imark, ilist);
    compact(PNonNeg{imark}, Ident{}, 0, nbad, wl, C_LIST1);
    int nst = fetch(C_LIST1);
    int *dw = dcount + C_LIST1;
    LAUNCH(k_fill, last_subseg, encl2, last_subseg, -1);
    LAUNCH(k_mark_onsegs, nst, M, wl, dw, sinks, encl2);
    int rc = ensure_slots(nst, 2 * nst);
    if (rc) return rc;
    LAUNCH(k_reset_steiner, nst, M, wl, dw, sinks);
    KL(k_bump_epoch, 1, 32)(fc);
    LAUNCH(k_insert_steiner, nst, M, wl, dw, sinks, center, pslots(), tslots(), &fc->epoch, dctr + 0);
    LAUNCH(k_update_steiner_nbrs, nst, M, wl, dw, sinks);
    consume_slots(nst, 2 * nst);
    rc = flip_flop(last_triangle);
    if (rc) return rc;
    LAUNCH(k_onsegs_to_enc, last_subseg, M, encl2, last_subseg);
    return GQM_OK;
  }

  // ---- output compaction (refine.cu:5758-6428) ----
  int compact_output() {
    NvtxRange nvtx("gqm:compact_output");
    // triangles
    compact(PTriLive{M.tst}, Ident{}, 0, last_triangle, tail, C_MISC);
    int newn = fetch(C_MISC);
    LAUNCH(k_newidx_init, last_triangle, M, newidx, last_triangle, newn, M.tst, (uint8_t)TS_NOTNULL, false);
    if (newn < last_triangle) {
      compact(PTriNull{M.tst}, Ident{}, 0, newn, emptyt, C_LIST0);
      compact(PTriLive{M.tst}, Ident{}, newn, last_triangle, tail, C_LIST1);
      LAUNCH(k_compact_tris_move, last_triangle - newn, M, tail, emptyt, dcount + C_LIST1, newidx);
      LAUNCH(k_fix_nbrs, newn, M, newidx, newn);
      LAUNCH(k_fix_s2t, last_subseg, M, newidx, last_subseg);
    }
    int ntri = newn;
    // points
    compact(PPtLive{M.ps}, Ident{}, 0, last_point, pnew, C_MISC);
    int newp = fetch(C_MISC);
    LAUNCH(k_newidx_init, last_point, M, pnew, last_point, newp, M.ps, (uint8_t)PS_DELETED, true);
    if (newp < last_point) {
      compact(PPtDeleted{M.ps}, Ident{}, 0, newp, emptyp, C_LIST0);
      compact(PPtLive{M.ps}, Ident{}, newp, last_point, tail, C_LIST1);
      LAUNCH(k_compact_pts_move, last_point - newp, M, tail, emptyp, dcount + C_LIST1, pnew);
      LAUNCH(k_fix_tri_vertices, ntri, M, pnew, ntri);
    }
    out_np = newp;
    out_nt = ntri;
    out_ns = last_subseg;
    return GQM_OK;
  }

  // ---- the whole refinement ----
  int run(const gqm_cdt_in *in, bool on_device, const gqm_options *opt) {
    NvtxRange nvtx("gqm:refine");
    int rc = setup(opt->device);
    if (rc) return rc;
    have_result = false;
    stats = gqm_stats{};
    status = 0;
    theta = opt->theta;
    mode = opt->mode ? 1 : 0;
    pred_mode = opt->predicates ? 1 : 0;
    placement = opt->placement == GQM_PLACE_LEARNED ? GQM_PLACE_LEARNED : GQM_PLACE_PLAIN;
    if (placement == GQM_PLACE_LEARNED) {
      if (!mlp_w && (dalloc(&mlp_w, kMlpW) || dalloc(&mlp_b, kMlpB))) return GQM_ERR_MEMORY;
      std::vector<uint16_t> hw(kMlpW);
      std::vector<float> hb(kMlpB);
      mlp_pack(opt->mlp, hw.data(), hb.data());
      cudaMemcpyAsync(mlp_w, hw.data(), sizeof(uint16_t) * kMlpW, cudaMemcpyHostToDevice, st);
      cudaMemcpyAsync(mlp_b, hb.data(), sizeof(float) * kMlpB, cudaMemcpyHostToDevice, st);
      if (cudaStreamSynchronize(st) != cudaSuccess) return GQM_ERR_CUDA;
    }
    max_rounds = opt->max_rounds > 0 ? opt->max_rounds : 1000000;
    offcenter = 0;
    double offc = 0.0;
    if (opt->insert_policy == GQM_OFFCENTER) {  // refine.cu:6555-6567
      offcenter = 1;
      double cg = cos(theta * GQM_PI / 180);
      offc = 0.475 * sqrt((1.0 + cg) / (1.0 - cg));
    }
    offconstant = (int)offc;  // splitTriangles takes an int (refine.cu:5132)
    int np = in->numberofpoints, nt = in->numberoftriangles, ns = in->numberofsegments;
    nseg_in = ns;
    pointblock = (int)(np * 0.5);
    triblock = 2 * pointblock;
    pcap = np + pointblock;
    tcap = nt + triblock;
#ifdef GQM_TEST_TIGHT_BUFFERS
    // test builds: physical buffers exactly the logical capacity, so every
    // growth step goes through the reallocation path
    rc = alloc_points(std::max<long>(pcap, pphys));
    if (rc) return rc;
    rc = alloc_tris(std::max<long>(tcap, tphys));
    if (rc) return rc;
#else
    rc = alloc_points(std::max<long>(pcap + 3L * pointblock, pphys));
    if (rc) return rc;
    rc = alloc_tris(std::max<long>(tcap + 4L * triblock, tphys));
    if (rc) return rc;
#endif
    rc = alloc_subsegs(std::max<long>(4L * ns + 1024, sphys));
    if (rc) return rc;
    // inputs
    const double *dpts;
    const int *dtri_in, *dnbr_in, *dseg_in;
    size_t need = sizeof(double) * 2 * np + sizeof(int) * (6L * nt + 2L * ns) + 256;
    if (!on_device) {
      if (need > dinput_bytes) {
        if (dinput) cudaFree(dinput);
        dinput = nullptr;
        dinput_bytes = 0;
        if (cudaMalloc((void **)&dinput, need) != cudaSuccess) {
          dinput = nullptr;
          return GQM_ERR_MEMORY;
        }
        dinput_bytes = need;
      }
      char *base = (char *)dinput;
      double *p0 = (double *)base;
      int *t0 = (int *)(base + sizeof(double) * 2 * np);
      int *n0 = t0 + 3L * nt;
      int *s0 = n0 + 3L * nt;
      // the caller's arrays are packed into pinned memory on the host's cores,
      // then uploaded with one copy
      if (grow_pinned(need)) return GQM_ERR_MEMORY;
      const size_t bp = sizeof(double) * 2 * np, bt = sizeof(int) * 3 * nt, bs = sizeof(int) * 2 * ns;
      host_copy({{h_stage, in->pointlist, bp}, {h_stage + bp, in->trianglelist, bt},
                 {h_stage + bp + bt, in->neighborlist, bt}, {h_stage + bp + 2 * bt, in->segmentlist, bs}});
      cudaMemcpyAsync(base, h_stage, bp + 2 * bt + bs, cudaMemcpyHostToDevice, st);
      dpts = p0;
      dtri_in = t0;
      dnbr_in = n0;
      dseg_in = s0;
    } else {
      dpts = in->pointlist;
      dtri_in = in->trianglelist;
      dnbr_in = in->neighborlist;
      dseg_in = in->segmentlist;
    }
    cudaEventRecord(ev0, st);
    if (grow_dev(&segs, &segs_cap, (size_t)ns + 1)) return GQM_ERR_MEMORY;
    if (ns) cudaMemcpyAsync(segs, dseg_in, sizeof(int2) * ns, cudaMemcpyDeviceToDevice, st);
    M.segs = segs;
    cudaMemsetAsync(M.s2t, 0, sizeof(s2t_t) * sphys, st);
    if (M.wbits) {  // left set only by a run that stopped inside a flip step
      cudaMemsetAsync(M.wbits, 0, sizeof(unsigned) * (tphys / 32 + 1), st);
      cudaMemsetAsync(M.wcnt, 0, sizeof(int) * (tphys / 1024 + 1), st);
      cudaMemsetAsync(M.wsup, 0, sizeof(int) * (tphys / 32768 + 1), st);
      cudaMemsetAsync(M.wmeg, 0, sizeof(int) * (tphys / 1048576 + 1), st);
    }
    cudaMemsetAsync(M.err, 0, sizeof(int), st);
    cudaMemsetAsync(dctr, 0, sizeof(unsigned long long) * 8, st);
    {
      const unsigned long long zero = 0;
      cudaMemcpyToSymbolAsync(g_incircle_fallbacks, &zero, sizeof(zero), 0, cudaMemcpyHostToDevice, st);
      // the small-step kernels' counters (their own translation units)
      gqm_fallbacks_cta(nullptr, 1, st);
      gqm_fallbacks_cluster(nullptr, 1, st);
    }
    KL(k_ctl_reset, 1, 32)(fc, 64 * max_rounds, M.err);
    LAUNCH(k_check_input, std::max(np, nt), (const double2 *)dpts, np, dtri_in, dnbr_in, nt, dseg_in, ns, M.err);
    rc = check_device_error();
    if (rc) return rc;
    // cos^2(theta) on the device, as the reference evaluates it
    KL(k_goodcos, 1, 32)(theta, dgc);
    double hgc[2];
    cudaMemcpyAsync(hgc, dgc, sizeof(double) * 2, cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    M.gc2 = hgc[0];
    M.mode = mode;
    M.max_area = opt->max_area > 0.0 ? opt->max_area : 0.0;
    stats.goodcos2 = hgc[0];
    LAUNCH(k_init_points, pphys, M, (const double2 *)dpts, np, (int)pphys);
    LAUNCH(k_init_tris, tphys, M, dtri_in, dnbr_in, nt, (int)tphys);
    // initSubsegs via a hash of segment endpoints
    {
      unsigned hsz = 1;
      while (hsz < 2u * (unsigned)ns + 16) hsz <<= 1;
      if (hsz > hash_cap) {  // the three tables share one capacity, set once all three exist
        hash_cap = 0;
        size_t c0 = 0, c1 = 0, c2 = 0;
        if (hvals) cudaFree(hvals);
        if (s2ti) cudaFree(s2ti);
        hvals = nullptr;
        s2ti = nullptr;
        if (grow_dev(&hkeys, &c0, hsz) || grow_dev(&hvals, &c1, hsz) || grow_dev(&s2ti, &c2, hsz))
          return GQM_ERR_MEMORY;
        hash_cap = hsz;
      }
      cudaMemsetAsync(hkeys, 0xff, sizeof(unsigned long long) * hsz, st);
      cudaMemsetAsync(s2ti, 0xff, sizeof(int) * (ns + 1), st);
      LAUNCH(k_seg_hash_insert, ns, segs, ns, hkeys, hvals, hsz - 1);
      LAUNCH(k_init_subsegs, nt, M, nt, hkeys, hvals, hsz - 1, s2ti);
      LAUNCH(k_pack_s2t, ns, M, s2ti, ns);
    }
    last_point = np;
    last_triangle = nt;
    last_subseg = ns;
    nempty_p = refresh_points();
    nempty_t = refresh_tris();
    LAUNCH(k_mark_all_encsegs, ns, M, ns);
    rc = split_encsegs();
    int rounds = 0;
    while (rc == 0) {
      LAUNCH(k_mark_bad, last_triangle, M, last_triangle);
      compact(PBad{M.tst}, Ident{}, 0, last_triangle, bad, C_LIST2);
      // the bad count and the device error word in one round trip
      cudaMemcpyAsync(hcount + C_LIST2, dcount + C_LIST2, sizeof(int), cudaMemcpyDeviceToHost, st);
      cudaMemcpyAsync(hcount + C_MISC, M.err, sizeof(int), cudaMemcpyDeviceToHost, st);
      if (cudaStreamSynchronize(st) != cudaSuccess) {
        rc = GQM_ERR_CUDA;
        break;
      }
      stats.host_syncs++;
      const int nbad = hcount[C_LIST2];
      const int derr = hcount[C_MISC];
      if (derr) {
        rc = derr;
        break;
      }
      if (nbad == 0) break;
      if (rounds >= max_rounds) {
        rc = GQM_ERR_ROUND_LIMIT;
        break;
      }
      stats.bad_total += nbad;
      rc = split_triangles(nbad);
      if (rc) break;
      rc = split_encsegs();
      if (rc) break;
      LAUNCH(k_points_old, last_point, M, last_point);
      rounds++;
    }
    stats.rounds = rounds;
    if (rc == 0) rc = check_device_error();
    if (rc == 0) rc = compact_output();
    cudaEventRecord(ev1, st);
    cudaError_t ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess) rc = GQM_ERR_CUDA;
    if (rc == 0) {
      int derr = check_device_error();
      if (derr) rc = derr;
    }
    float ms = 0;
    cudaEventElapsedTime(&ms, ev0, ev1);
    stats.device_ms = ms;
    collect_loop_events();
    unsigned long long hc[8];
    cudaMemcpy(hc, dctr, sizeof(hc), cudaMemcpyDeviceToHost);
    stats.learned_candidates = (long long)hc[4];
    stats.learned_used = (long long)hc[5];
    FlipCtl hf;
    cudaMemcpy(&hf, fc, sizeof(hf), cudaMemcpyDeviceToHost);
    stats.flip_steps = hf.steps;
    // each graph launch counted one kernel (its loop-entry kernel); the nine
    // kernels of every loop iteration it ran (a grid step, its condition and
    // the single-block kernel that runs the small steps after it) are added here
    if (use_graph) stats.kernel_launches += (long long)step_kernels() * (hf.steps - hf.small_steps);
    for (int b = 0; b < kFlipProfileBins; ++b) {
      flip_prof_steps[b] = (long long)hf.prof_steps[b];
      flip_prof_items[b] = (long long)hf.prof_items[b];
    }
    stats.steiner_inserted = (long long)hc[0];
    stats.midpoints_inserted = (long long)hc[1];
    {
      unsigned long long fb = 0;
      cudaMemcpyFromSymbol(&fb, g_incircle_fallbacks, sizeof(fb));
      gqm_fallbacks_cta(&fb, 0, st);
      gqm_fallbacks_cluster(&fb, 0, st);
      stats.exact_fallbacks = (long long)fb;
    }
    have_result = (rc == 0);
    status = rc;
    return rc;
  }

  int result(gqm_cdt_out *out) {
    NvtxRange nvtx("gqm:result");
    if (!have_result) return GQM_ERR_ARGUMENT;
    memset(out, 0, sizeof(*out));
    const long np = out_np, nt = out_nt, ns = out_ns;
    // one block on the device: points | triangles | neighbours | segments |
    // point status | triangle status, each on 16 bytes; one download into
    // pinned memory, then copies into the caller's arrays on the host's cores
    auto up16 = [](size_t x) { return (x + 15) & ~(size_t)15; };
    const size_t o_tri = up16(16 * (size_t)np), o_nbr = o_tri + up16(12 * (size_t)nt),
                 o_seg = o_nbr + up16(12 * (size_t)nt), o_ps = o_seg + up16(8 * (size_t)ns),
                 o_ts = o_ps + up16((size_t)np), bytes = o_ts + up16((size_t)nt);
    if (grow_dev(&d_out, &d_out_cap, bytes) || grow_pinned(bytes)) return GQM_ERR_MEMORY;
    cudaMemcpyAsync(d_out, M.pts, 16 * (size_t)np, cudaMemcpyDeviceToDevice, st);
    LAUNCH(k_emit_output, std::max(nt, ns), M, (int)nt, (int)ns, (int *)(d_out + o_tri), (int *)(d_out + o_nbr),
           (int *)(d_out + o_seg), (uint8_t *)(d_out + o_ts));
    LAUNCH(k_emit_pstatus, np, M, (int)np, (uint8_t *)(d_out + o_ps));
    cudaMemcpyAsync(h_stage, d_out, bytes, cudaMemcpyDeviceToHost, st);
    out->numberofpoints = (int)np;
    out->numberoftriangles = (int)nt;
    out->numberofsegments = (int)ns;
    out->pointlist = (double *)malloc(sizeof(double) * 2 * (size_t)np + 16);
    out->trianglelist = (int *)malloc(sizeof(int) * 3 * (size_t)nt + 16);
    out->neighborlist = (int *)malloc(sizeof(int) * 3 * (size_t)nt + 16);
    out->segmentlist = (int *)malloc(sizeof(int) * 2 * (size_t)ns + 16);
    out->pstatus = (unsigned char *)malloc((size_t)np + 16);
    out->tstatus = (unsigned char *)malloc((size_t)nt + 16);
    advise_huge(out->pointlist, 16 * (size_t)np);
    advise_huge(out->trianglelist, 12 * (size_t)nt);
    advise_huge(out->neighborlist, 12 * (size_t)nt);
    advise_huge(out->tstatus, (size_t)nt);
    const cudaError_t ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess || !out->pointlist || !out->trianglelist || !out->neighborlist || !out->segmentlist ||
        !out->pstatus || !out->tstatus) {
      for (void *q : {(void *)out->pointlist, (void *)out->trianglelist, (void *)out->neighborlist,
                      (void *)out->segmentlist, (void *)out->pstatus, (void *)out->tstatus})
        free(q);
      memset(out, 0, sizeof(*out));
      return ce != cudaSuccess ? GQM_ERR_CUDA : GQM_ERR_MEMORY;
    }
    host_copy({{out->pointlist, h_stage, 16 * (size_t)np}, {out->trianglelist, h_stage + o_tri, 12 * (size_t)nt},
               {out->neighborlist, h_stage + o_nbr, 12 * (size_t)nt}, {out->segmentlist, h_stage + o_seg, 8 * (size_t)ns},
               {out->pstatus, h_stage + o_ps, (size_t)np}, {out->tstatus, h_stage + o_ts, (size_t)nt}});
    return GQM_OK;
  }
};

}  // namespace gqm

struct gqm_context {
  gqm::Refiner r;
};

extern "C" {

void gqm_default_options(gqm_options *o) {
  o->theta = 20.0;
  o->insert_policy = GQM_OFFCENTER;
  o->mode = GQM_RUPPERT;
  o->predicates = GQM_PRED_REFERENCE;
  o->device = 0;
  o->max_rounds = 0;
  o->placement = GQM_PLACE_PLAIN;
  o->mlp = nullptr;
  o->max_area = 0.0;
}

static int validate(const gqm_cdt_in *in, const gqm_options *opt) {
  if (!in || !opt) return GQM_ERR_ARGUMENT;
  if (in->numberofpoints < 3 || in->numberoftriangles < 1 || in->numberofsegments < 0) return GQM_ERR_ARGUMENT;
  if (!in->pointlist || !in->trianglelist || !in->neighborlist) return GQM_ERR_ARGUMENT;
  if (in->numberofsegments > 0 && !in->segmentlist) return GQM_ERR_ARGUMENT;
  if (!(opt->theta > 0.0 && opt->theta < 60.0)) return GQM_ERR_ARGUMENT;
  if (opt->placement != GQM_PLACE_PLAIN && (opt->placement != GQM_PLACE_LEARNED || !opt->mlp)) return GQM_ERR_ARGUMENT;
  if (!(opt->max_area >= 0.0)) return GQM_ERR_ARGUMENT;
  return GQM_OK;
}

int gqm_context_create(int device, gqm_context **ctx) {
  if (!ctx) return GQM_ERR_ARGUMENT;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= device || device < 0) return GQM_ERR_NO_DEVICE;
  *ctx = new gqm_context();
  int rc = (*ctx)->r.setup(device);
  if (rc) {
    delete *ctx;
    *ctx = nullptr;
  }
  return rc;
}
void gqm_context_destroy(gqm_context *ctx) { delete ctx; }
int gqm_context_run(gqm_context *ctx, const gqm_cdt_in *in, int in_on_device, const gqm_options *opt,
                    gqm_stats *stats) {
  if (!ctx) return GQM_ERR_ARGUMENT;
  int rc = validate(in, opt);
  if (rc) return rc;
  rc = ctx->r.run(in, in_on_device != 0, opt);
  if (stats) *stats = ctx->r.stats;
  return rc;
}
int gqm_context_result(gqm_context *ctx, gqm_cdt_out *out) {
  if (!ctx || !out) return GQM_ERR_ARGUMENT;
  return ctx->r.result(out);
}
int gqm_context_probe(gqm_context *ctx, int enable) {
  if (!ctx || !ctx->r.ktm) return GQM_ERR_ARGUMENT;
  gqm::Refiner &r = ctx->r;
  if (cudaSetDevice(r.device) != cudaSuccess) return GQM_ERR_CUDA;
#ifdef GQM_HOST_EMU
  gqm::k_ktimer_reset(r.ktm, enable ? 1 : 0);
  gqm::k_ktimer_reset(r.stm, enable ? 1 : 0);
#else
  gqm::k_ktimer_reset<<<1, 32, 0, r.st>>>(r.ktm, enable ? 1 : 0);
  gqm::k_ktimer_reset<<<1, 32, 0, r.st>>>(r.stm, enable ? 1 : 0);
#endif
  r.probing = enable != 0;
  r.probe_loop_ms = 0.0;
  r.probe_loops = 0;
  return cudaStreamSynchronize(r.st) == cudaSuccess ? GQM_OK : GQM_ERR_CUDA;
}
int gqm_context_probe_read(gqm_context *ctx, gqm_probe *p) {
  if (!ctx || !p || !ctx->r.ktm) return GQM_ERR_ARGUMENT;
  gqm::Refiner &r = ctx->r;
  if (cudaSetDevice(r.device) != cudaSuccess) return GQM_ERR_CUDA;
  gqm::KTimer h, hs;
  if (cudaStreamSynchronize(r.st) != cudaSuccess ||
      cudaMemcpy(&h, r.ktm, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(&hs, r.stm, sizeof(hs), cudaMemcpyDeviceToHost) != cudaSuccess)
    return GQM_ERR_CUDA;
  p->small_launches = (long long)hs.launches;
  p->small_items = (long long)hs.items;
  p->small_winners = (long long)hs.winners;
  p->small_ms = (double)hs.total_ns * 1e-6;
  p->check_launches = (long long)h.launches;
  p->check_items = (long long)h.items;
  p->check_ms = (double)h.total_ns * 1e-6;
  for (int i = 0; i < 4; ++i) p->first_items[i] = (long long)h.first_items[i];
  p->loop_launches = r.probe_loops;
  p->loop_ms = r.probe_loop_ms;
  return GQM_OK;
}
int gqm_context_set_tuning(gqm_context *ctx, const gqm_tuning *t) {
  if (!ctx || !t) return GQM_ERR_ARGUMENT;
  gqm::Refiner::Tuning n;
  if (t->step_grid < 0 || t->step_grid > 148 * 64) return GQM_ERR_ARGUMENT;
  if (t->step_grid > 0) n.step_grid = t->step_grid;
  if (t->small_limit < 0)
    n.small_limit = 0;
  else if (t->small_limit > 0)
    n.small_limit = t->small_limit;
  if (t->small_cluster != 0 && t->small_cluster != 1 && t->small_cluster != 8 && t->small_cluster != 16)
    return GQM_ERR_ARGUMENT;
  if (t->small_cluster > 1) n.small_cluster = t->small_cluster;
  if (t->check_blocks_per_sm < 0 || t->check_blocks_per_sm > 2) return GQM_ERR_ARGUMENT;
  if (t->check_blocks_per_sm > 0) n.check_minb = t->check_blocks_per_sm;
  if (n.small_cluster > 1) {
    if (cudaSetDevice(ctx->r.device) != cudaSuccess) return GQM_ERR_CUDA;
    if (!gqm_flip_cluster_ok(n.small_cluster)) return GQM_ERR_CUDA;
  }
  ctx->r.tune = n;
  return GQM_OK;
}
int gqm_context_get_tuning(gqm_context *ctx, gqm_tuning *t) {
  if (!ctx || !t) return GQM_ERR_ARGUMENT;
  const gqm::Refiner::Tuning &c = ctx->r.tune;
  t->step_grid = c.step_grid;
  t->small_limit = c.small_limit > 0 ? c.small_limit : -1;
  t->small_cluster = c.small_cluster;
  t->check_blocks_per_sm = c.check_minb;
  return GQM_OK;
}
int gqm_context_autotune(gqm_context *ctx, const gqm_cdt_in *in, int in_on_device, const gqm_options *opt,
                         int repeats, gqm_tuning *chosen, double *best_ms) {
  if (!ctx || !chosen) return GQM_ERR_ARGUMENT;
  int rc = validate(in, opt);
  if (rc) return rc;
  if (repeats < 1) repeats = 1;
  gqm::Refiner &R = ctx->r;
  auto time_of = [&](double *ms) -> int {
    double best = 1e300;
    for (int k = 0; k < repeats; ++k) {
      int e = R.run(in, in_on_device != 0, opt);
      if (e) return e;
      best = std::min(best, (double)R.stats.device_ms);
    }
    *ms = best;
    return GQM_OK;
  };
  gqm_tuning cur;
  gqm_context_get_tuning(ctx, &cur);
  // one untimed run first: buffers grow and the loop graph is built once
  rc = R.run(in, in_on_device != 0, opt);
  if (rc) return rc;
  double best = 0.0;
  rc = time_of(&best);
  if (rc) return rc;
  // one field at a time, in order of expected effect; each candidate that the
  // device cannot run (a cluster size it cannot place) is skipped
  const int checks[] = {2, 1};
  const int clusters[] = {1, 8, 16};
  const int limits[] = {512, 1024, 2048, 4096};
  const int grids[] = {148 * 2, 148 * 4, 148 * 8};
  for (int field = 0; field < 4; ++field) {
    const int *vals = field == 0 ? checks : field == 1 ? clusters : field == 2 ? limits : grids;
    const int nv = field == 0 ? 2 : field == 1 ? 3 : field == 2 ? 4 : 3;
    for (int k = 0; k < nv; ++k) {
      gqm_tuning cand = cur;
      int *f = field == 0 ? &cand.check_blocks_per_sm
                          : field == 1 ? &cand.small_cluster : field == 2 ? &cand.small_limit : &cand.step_grid;
      if (*f == vals[k]) continue;
      *f = vals[k];
      if (gqm_context_set_tuning(ctx, &cand) != GQM_OK) continue;
      double ms = 0.0;
      rc = time_of(&ms);
      if (rc) {
        gqm_context_set_tuning(ctx, &cur);
        return rc;
      }
      if (ms < best) {
        best = ms;
        cur = cand;
      }
    }
    gqm_context_set_tuning(ctx, &cur);
  }
  gqm_context_get_tuning(ctx, chosen);
  if (best_ms) *best_ms = best;
  return GQM_OK;
}
int gqm_context_flip_profile(gqm_context *ctx, long long *steps, long long *items) {
  if (!ctx || !steps || !items) return GQM_ERR_ARGUMENT;
  for (int b = 0; b < gqm::kFlipProfileBins; ++b) {
    steps[b] = ctx->r.flip_prof_steps[b];
    items[b] = ctx->r.flip_prof_items[b];
  }
  return GQM_OK;
}
int gqm_learn_collect(const gqm_cdt_in *in, const gqm_options *opt, float *features, float *targets, long long cap,
                      long long *count) {
  if (!in || !opt || cap < 0 || (cap > 0 && (!features || !targets))) return GQM_ERR_ARGUMENT;
  gqm_options o = *opt;
  o.placement = GQM_PLACE_PLAIN;  // the rows describe the plain refinement
  o.mlp = nullptr;
  int rc = validate(in, &o);
  if (rc) return rc;
  gqm_context *ctx = nullptr;
  rc = gqm_context_create(o.device, &ctx);
  if (rc) return rc;
  gqm::Refiner &r = ctx->r;
  const size_t rows = (size_t)(cap > 0 ? cap : 1);
  if (r.dalloc(&r.col_feat, rows * gqm::kFeat) || r.dalloc(&r.col_tgt, rows) || r.dalloc(&r.col_cnt, 1)) {
    rc = GQM_ERR_MEMORY;
  } else {
    cudaMemset(r.col_cnt, 0, sizeof(unsigned long long));
    r.col_cap = (unsigned long long)cap;
    gqm_stats st;
    rc = gqm_context_run(ctx, in, 0, &o, &st);
    unsigned long long n = 0;
    if (!rc && cudaMemcpy(&n, r.col_cnt, sizeof(n), cudaMemcpyDeviceToHost) != cudaSuccess) rc = GQM_ERR_CUDA;
    if (!rc) {
      const long long m = (long long)std::min<unsigned long long>(n, (unsigned long long)cap);
      if (m > 0 && (cudaMemcpy(features, r.col_feat, sizeof(float) * gqm::kFeat * m, cudaMemcpyDeviceToHost) !=
                        cudaSuccess ||
                    cudaMemcpy(targets, r.col_tgt, sizeof(float) * m, cudaMemcpyDeviceToHost) != cudaSuccess))
        rc = GQM_ERR_CUDA;
      if (count) *count = m;
    }
  }
  if (r.col_feat) cudaFree(r.col_feat);
  if (r.col_tgt) cudaFree(r.col_tgt);
  if (r.col_cnt) cudaFree(r.col_cnt);
  r.col_feat = r.col_tgt = nullptr;
  r.col_cnt = nullptr;
  gqm_context_destroy(ctx);
  return rc;
}
int gqm_context_result_sizes(gqm_context *ctx, int *np, int *nt, int *ns) {
  if (!ctx || !ctx->r.have_result) return GQM_ERR_ARGUMENT;
  if (np) *np = ctx->r.out_np;
  if (nt) *nt = ctx->r.out_nt;
  if (ns) *ns = ctx->r.out_ns;
  return GQM_OK;
}
void *gqm_context_stream(gqm_context *ctx) { return ctx ? (void *)ctx->r.st : nullptr; }

// One cached context per device for gqm_refine: device buffers and the
// captured flip-loop graph are reused by later calls instead of being
// allocated every time.  Callers hold g_cache_mutex.
static std::mutex g_cache_mutex;
static gqm_context *g_cache[64] = {};
static int cached_context(int device, gqm_context **out) {
  gqm_context *&ctx = g_cache[device];
  if (!ctx) {
    int rc = gqm_context_create(device, &ctx);
    if (rc) return rc;
  }
  *out = ctx;
  return GQM_OK;
}

int gqm_refine(const gqm_cdt_in *in, gqm_cdt_out *out, const gqm_options *opt, gqm_stats *stats) {
  if (!out) return GQM_ERR_ARGUMENT;
  memset(out, 0, sizeof(*out));
  gqm_options def;
  if (!opt) {
    gqm_default_options(&def);
    opt = &def;
  }
  int rc = validate(in, opt);
  if (rc) return rc;
  if (opt->device < 0 || opt->device >= 64) return GQM_ERR_NO_DEVICE;
  std::lock_guard<std::mutex> lock(g_cache_mutex);
  gqm_context *ctx = nullptr;
  rc = cached_context(opt->device, &ctx);
  if (rc) return rc;
  rc = gqm_context_run(ctx, in, 0, opt, stats);
  if (rc == GQM_OK) rc = gqm_context_result(ctx, out);
  return rc;
}

int gqm_set_default_tuning(int device, const gqm_tuning *t) {
  if (!t || device < 0 || device >= 64) return GQM_ERR_ARGUMENT;
  std::lock_guard<std::mutex> lock(g_cache_mutex);
  gqm_context *ctx = nullptr;
  int rc = cached_context(device, &ctx);
  if (rc) return rc;
  return gqm_context_set_tuning(ctx, t);
}

int gqm_refine_batch(int ndomains, const gqm_cdt_in *in, gqm_cdt_out *out, const gqm_options *opt,
                     gqm_stats *stats, int workers, int *failed_domain) {
  if (failed_domain) *failed_domain = -1;
  if (ndomains < 0 || (ndomains > 0 && (!in || !out || !opt))) return GQM_ERR_ARGUMENT;
  for (int i = 0; i < ndomains; ++i) memset(&out[i], 0, sizeof(gqm_cdt_out));
  if (ndomains == 0) return GQM_OK;
  for (int i = 0; i < ndomains; ++i) {
    int rc = validate(&in[i], &opt[i]);
    if (rc) {
      if (failed_domain) *failed_domain = i;
      return rc;
    }
  }
  if (workers < 1) workers = 1;
  if (workers > ndomains) workers = ndomains;
  // largest domains first (longest-processing-time order)
  std::vector<int> order(ndomains);
  for (int i = 0; i < ndomains; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return in[a].numberofpoints > in[b].numberofpoints; });
  std::atomic<int> next(0), first_err(0), err_dom(-1);
  auto work = [&](int) {
    gqm_context *ctx = nullptr;
    for (;;) {
      int k = next.fetch_add(1);
      if (k >= ndomains || first_err.load() != 0) break;
      int d = order[k];
      int rc = GQM_OK;
      if (!ctx) rc = gqm_context_create(opt[d].device, &ctx);
      gqm_stats st;
      if (rc == GQM_OK) rc = gqm_context_run(ctx, &in[d], 0, &opt[d], &st);
      if (rc == GQM_OK) rc = gqm_context_result(ctx, &out[d]);
      if (rc == GQM_OK && stats) stats[d] = st;
      if (rc != GQM_OK) {
        int zero = 0;
        if (first_err.compare_exchange_strong(zero, rc)) err_dom.store(d);
      }
    }
    if (ctx) gqm_context_destroy(ctx);
  };
  std::vector<std::thread> pool;
  for (int w = 0; w < workers; ++w) pool.emplace_back(work, w);
  for (auto &t : pool) t.join();
  if (failed_domain) *failed_domain = err_dom.load();
  return first_err.load();
}

void gqm_free_result(gqm_cdt_out *out) {
  if (!out) return;
  free(out->pointlist);
  free(out->trianglelist);
  free(out->neighborlist);
  free(out->segmentlist);
  free(out->pstatus);
  free(out->tstatus);
  memset(out, 0, sizeof(*out));
}

const char *gqm_status_string(int s) {
  switch (s) {
    case GQM_OK: return "ok";
    case GQM_ERR_ARGUMENT: return "invalid argument";
    case GQM_ERR_ROUND_LIMIT: return "refinement loop exceeded max_rounds";
    case GQM_ERR_WALK_LIMIT: return "point location walk did not end";
    case GQM_ERR_FAN_LIMIT: return "vertex fan walk did not close";
    case GQM_ERR_TOPOLOGY: return "mesh inconsistency";
    case GQM_ERR_CAVITY: return "cavity walk exceeded its bound";
    case GQM_ERR_CUDA: return "CUDA runtime error";
    case GQM_ERR_NO_DEVICE: return "no CUDA device";
    case GQM_ERR_MEMORY: return "device allocation failed";
    case GQM_ERR_INPUT_CDT: return "the CDT of the points and segments could not be built";
    case GQM_ERR_ARENA: return "a batched domain outgrew its scratch arena";
    case GQM_ERR_TOO_LARGE: return "result larger than the no-allocation staging array";
    default: return "unknown status";
  }
}
int gqm_version(void) { return 101; }
#ifndef GQM_CONTRACTED
#define GQM_CONTRACTED 0
#endif
int gqm_arithmetic(void) { return GQM_CONTRACTED ? GQM_ARITH_CONTRACTED : GQM_ARITH_SEPARATE; }

}  // extern "C"

// ============================================================================
// Result copy without allocation (gqm_context_result_noalloc).
//
// For callers that cannot allocate at the time they read a result: a service
// with a device memory budget fixed at start-up that reads many small results
// in a loop, or code sharing the GPU with work that must not be stalled by the
// device-wide synchronization a cudaFree implies.  gqm_context_result() mallocs
// the host result arrays on every call and grows its device and pinned staging
// buffers (cudaMalloc / cudaFree) whenever a larger result arrives; the kernel
// below is its result-emission kernel staging into a statically allocated
// device array instead, and the caller provides the host arrays.
// ============================================================================
namespace gqm {

constexpr int kNoAllocRows = GQM_NOALLOC_MAX_ELEMENTS;
// Staging layout (bytes): triangles 3 ints, neighbours 3 ints, segments
// 2 ints, triangle status 1 byte, point status 1 byte per row.
constexpr size_t kNoAllocTri = 0;
constexpr size_t kNoAllocNbr = kNoAllocTri + sizeof(int) * 3 * kNoAllocRows;
constexpr size_t kNoAllocSeg = kNoAllocNbr + sizeof(int) * 3 * kNoAllocRows;
constexpr size_t kNoAllocTs = kNoAllocSeg + sizeof(int) * 2 * kNoAllocRows;
constexpr size_t kNoAllocPs = kNoAllocTs + (size_t)kNoAllocRows;
constexpr size_t kNoAllocBytes = kNoAllocPs + (size_t)kNoAllocRows;

// One array per device, held until the process exits; shared by every call.
static __device__ __align__(256) unsigned char g_noalloc_staging[kNoAllocBytes];

// Device address of g_noalloc_staging per device ordinal.  In host code the
// array's name is only a host-side handle, so the address is looked up once
// per device, with that device current, and then passed to the kernel.
static unsigned char *g_noalloc_addr[64];
static bool g_noalloc_ready[64];
static std::mutex g_noalloc_mutex;

static int noalloc_staging(int device, unsigned char **p) {
  if (device < 0 || device >= 64) return GQM_ERR_NO_DEVICE;
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ready[device]) {
    void *addr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&addr, g_noalloc_staging);
    if (e != cudaSuccess || addr == nullptr) return GQM_ERR_CUDA;
    g_noalloc_addr[device] = (unsigned char *)addr;
    g_noalloc_ready[device] = true;
  }
  *p = g_noalloc_addr[device];
  return GQM_OK;
}

// k_emit_output / k_emit_pstatus writing into the staging array.  Every row
// that is copied out is written first, so nothing has to start at zero.
__global__ void k_emit_output_staged(Mesh M, int np, int nt, int ns, unsigned char *stage) {
  int *tri = reinterpret_cast<int *>(stage + kNoAllocTri);
  int *nbr = reinterpret_cast<int *>(stage + kNoAllocNbr);
  int *seg = reinterpret_cast<int *>(stage + kNoAllocSeg);
  uint8_t *ts = stage + kNoAllocTs;
  uint8_t *ps = stage + kNoAllocPs;
  GS_LOOP(i, max(max(nt, ns), np)) {
    if (i < nt) {
      int4 v = M.tv[i], nb = M.tn[i];
      tri[3 * i] = v.x;
      tri[3 * i + 1] = v.y;
      tri[3 * i + 2] = v.z;
      nbr[3 * i] = dtri(nb.x);
      nbr[3 * i + 1] = dtri(nb.y);
      nbr[3 * i + 2] = dtri(nb.z);
      ts[i] = (uint8_t)((M.tst[i] & 7) | (M.tflip[i] ? 8 : 0) | (M.tfo[i] << 4));
    }
    if (i < ns) {
      int o = s2t_get(M, i);
      if (o < 0) {
        seg[2 * i] = seg[2 * i + 1] = -1;
      } else {
        int4 v = M.tv[dtri(o)];
        int r = dori(o);
        seg[2 * i] = comp(v, m3(r + 1));
        seg[2 * i + 1] = comp(v, m3(r + 2));
      }
    }
    if (i < np) ps[i] = (uint8_t)((M.ps[i] & 15) | (M.pred[i] ? 16 : 0));
  }
}

}  // namespace gqm

extern "C" int gqm_context_result_noalloc(gqm_context *ctx, gqm_cdt_out *out) {
  if (!ctx || !out || !ctx->r.have_result) return GQM_ERR_ARGUMENT;
  gqm::Refiner &R = ctx->r;
  int np = R.out_np, nt = R.out_nt, ns = R.out_ns;
  if (np > gqm::kNoAllocRows || nt > gqm::kNoAllocRows || ns > gqm::kNoAllocRows) return GQM_ERR_TOO_LARGE;
  if (!out->pointlist || !out->trianglelist || !out->neighborlist || !out->segmentlist || !out->pstatus ||
      !out->tstatus)
    return GQM_ERR_ARGUMENT;
  if (cudaSetDevice(R.device) != cudaSuccess) return GQM_ERR_CUDA;
  unsigned char *stage = nullptr;
  int rc = gqm::noalloc_staging(R.device, &stage);
  if (rc) return rc;
  cudaStream_t st = R.st;
  int work = std::max(std::max(nt, ns), np);
  KL(gqm::k_emit_output_staged, gqm::Refiner::grid_for(work), 256)(R.M, np, nt, ns, stage);
  if (cudaGetLastError() != cudaSuccess) return GQM_ERR_CUDA;
  // errors reported when a copy is issued (an invalid host pointer, for one)
  // are not sticky, so each copy's status is checked here: a failed call
  // returns before the counts are written
  const struct {
    void *dst;
    const void *src;
    size_t bytes;
  } copies[] = {{out->pointlist, R.M.pts, sizeof(double) * 2 * (size_t)np},
                {out->trianglelist, stage + gqm::kNoAllocTri, sizeof(int) * 3 * (size_t)nt},
                {out->neighborlist, stage + gqm::kNoAllocNbr, sizeof(int) * 3 * (size_t)nt},
                {out->segmentlist, stage + gqm::kNoAllocSeg, sizeof(int) * 2 * (size_t)ns},
                {out->tstatus, stage + gqm::kNoAllocTs, (size_t)nt},
                {out->pstatus, stage + gqm::kNoAllocPs, (size_t)np}};
  for (const auto &c : copies)
    if (cudaMemcpyAsync(c.dst, c.src, c.bytes, cudaMemcpyDeviceToHost, st) != cudaSuccess) {
      cudaStreamSynchronize(st);  // copies already issued finish before the caller reuses its arrays
      return GQM_ERR_CUDA;
    }
  if (cudaStreamSynchronize(st) != cudaSuccess) return GQM_ERR_CUDA;
  out->numberofpoints = np;
  out->numberoftriangles = nt;
  out->numberofsegments = ns;
  return GQM_OK;
}
