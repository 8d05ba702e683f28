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
#include <climits>
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
// Pinned blocks for large results.  A result of gqm_refine /
// gqm_context_result of at least kPoolMinBytes, and the results of a
// persistent batch together, are downloaded straight into a block of pinned
// host memory that the callers then own until gqm_free_result, which gives
// their share back (a batch's block is shared by its domains and is free again
// once every domain's result is released): no second copy from a staging
// buffer and no page faults on fresh memory.  The pool holds at most
// kPoolMaxBytes; when no block fits and the limit is reached, the result takes
// the malloc path (staging buffer, then copies).
// ============================================================================
constexpr size_t kPoolMinBytes = 16ull << 20;
constexpr size_t kPoolMaxBytes = 8ull << 30;
struct PoolBlock {
  char *p;
  size_t cap;
  int refs;  // results still holding the block (0: free)
};
static std::mutex g_pool_mutex;
static std::vector<PoolBlock> g_pool;
static size_t g_pool_bytes = 0;
}  // namespace gqm
// a block of at least `bytes` held by `refs` results, or nullptr
char *gqm_pinned_take(size_t bytes, int refs) {
  using namespace gqm;
  if (bytes < kPoolMinBytes || refs <= 0) return nullptr;
  std::lock_guard<std::mutex> lock(g_pool_mutex);
  PoolBlock *best = nullptr;
  for (PoolBlock &b : g_pool)
    if (!b.refs && b.cap >= bytes && (!best || b.cap < best->cap)) best = &b;
  if (best) {
    best->refs = refs;
    return best->p;
  }
  // make room: drop free blocks, which are all too small
  for (size_t k = 0; k < g_pool.size() && g_pool_bytes + bytes > kPoolMaxBytes;) {
    if (!g_pool[k].refs) {
      cudaFreeHost(g_pool[k].p);
      g_pool_bytes -= g_pool[k].cap;
      g_pool.erase(g_pool.begin() + (long)k);
    } else {
      ++k;
    }
  }
  if (g_pool_bytes + bytes > kPoolMaxBytes) return nullptr;
  char *p = nullptr;
  if (cudaMallocHost((void **)&p, bytes) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  g_pool.push_back(PoolBlock{p, bytes, refs});
  g_pool_bytes += bytes;
  return p;
}
// true when p lies in a lent pool block (whose count of holders drops by one)
bool gqm_pinned_give(const void *p) {
  using namespace gqm;
  if (!p) return false;
  const char *q = static_cast<const char *>(p);
  std::lock_guard<std::mutex> lock(g_pool_mutex);
  for (PoolBlock &b : g_pool)
    if (b.refs > 0 && q >= b.p && q < b.p + b.cap) {
      --b.refs;
      return true;
    }
  return false;
}
namespace gqm {
static char *pool_take(size_t bytes) { return gqm_pinned_take(bytes, 1); }
static bool pool_give(const void *p) { return gqm_pinned_give(p); }

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
// The driver's state on the device.  The reference keeps its bookkeeping of
// free slots (refine.cu:149-197, 3408-3444, 3545-3562, 5259-5296, 5354-5368)
// and every count it branches on in host variables; here they live in one
// DState block on the device, updated by one-thread kernels between the
// steps, so that the whole refinement (the splitting of encroached
// subsegments and the round loop, refine.cu:6830-7024) runs as one CUDA graph
// whose loops and branches are conditional nodes decided on the device.
// ============================================================================
constexpr int kMaxNodes = 40;  // conditional nodes of the refinement graph
struct DState {
  int pcap, tcap;                  // the reference's logical capacities of points / triangles
  int pphys, tphys, sphys, cav_cap;  // physical capacities of the buffers
  int last_point, last_triangle, last_subseg;
  int pointblock, triblock;
  int nempty_p, nempty_t, lenp, lent;
  int pslot, tslot;  // first free slot of the current batch: lenp - nempty_p, lent - nempty_t
  int req_p, req_t, grew;  // the batch's request; whether a growth step happened
  int nenc, nmark, ndel, nmid, nbad, nst;
  // a physical capacity would be exceeded (1 points, 2 triangles, 4
  // subsegments, 8 stored cavities): every loop ends and the host repeats the
  // run with larger buffers (the result does not depend on them)
  int need_grow;
  int flag;  // value of the last condition (read by the host when no graph runs)
  long long max_rounds, rounds, outer, inner, mid_iter, bad_total;
  long long iters[kMaxNodes + 1];  // runs of each conditional node's body
};

// one-thread kernels of the driver: f(DState &, int *err) changes the state
// (k_do) or returns a loop / branch condition (k_cond, which also sets the
// graph's conditional handle when the graph runs)
template <class F>
__global__ void k_do(F f, DState *d, int *err) {
  if (threadIdx.x == 0 && blockIdx.x == 0) f(*d, err);
}
template <class F>
__global__ void k_cond(F f, DState *d, int *err, cudaGraphConditionalHandle h, int graph, int node) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    const int v = f(*d, err) ? 1 : 0;
    d->flag = v;
    if (v) d->iters[node]++;
#ifndef GQM_HOST_EMU
    if (graph) cudaGraphSetConditional(h, v);
#endif
    (void)h;
    (void)graph;
  }
}
__device__ __forceinline__ bool run_ok(const DState &d, const int *err) { return *err == 0 && d.need_grow == 0; }

// splitEncsegs' outer loop (refine.cu:3180-3778): encroached subsegments remain
struct CondEncroached {
  __device__ bool operator()(DState &d, int *err) const {
    if (!run_ok(d, err) || d.nenc == 0) return false;
    if (++d.outer > d.max_rounds) {
      atomicCAS(err, 0, GQM_ERR_ROUND_LIMIT);
      return false;
    }
    d.nmark = d.nenc;
    d.inner = 0;
    d.mid_iter = 0;
    return true;
  }
};
// its deletion of free Steiner points inside diametral circles
struct CondDelete {
  __device__ bool operator()(DState &d, int *err) const {
    if (!run_ok(d, err) || d.ndel == 0) return false;
    if (++d.inner > d.max_rounds) {
      atomicCAS(err, 0, GQM_ERR_ROUND_LIMIT);
      return false;
    }
    d.nmark = d.ndel;
    return true;
  }
};
// its midpoint insertion passes
struct CondMidpoints {
  __device__ bool operator()(DState &d, int *err) const {
    if (!run_ok(d, err) || d.nmid == 0) return false;
    if (++d.mid_iter > 64 * d.max_rounds) {
      atomicCAS(err, 0, GQM_ERR_ROUND_LIMIT);
      return false;
    }
    return true;
  }
};
// the round loop (refine.cu:6830-7024): bad triangles remain
struct CondRound {
  __device__ bool operator()(DState &d, int *err) const {
    if (!run_ok(d, err) || d.nbad == 0) return false;
    if (d.rounds >= d.max_rounds) {
      atomicCAS(err, 0, GQM_ERR_ROUND_LIMIT);
      return false;
    }
    d.bad_total += d.nbad;
    return true;
  }
};
// the growth steps of refine.cu:3408-3444 / 5259-5296
struct CondNeedPoints {
  __device__ bool operator()(DState &d, int *err) const { return run_ok(d, err) && d.req_p > d.nempty_p; }
};
struct CondNeedTris {
  __device__ bool operator()(DState &d, int *err) const { return run_ok(d, err) && d.req_t > d.nempty_t; }
};
struct CondGrew {
  __device__ bool operator()(DState &d, int *) const { return d.grew != 0; }
};
struct SlotsRequest {  // a batch of *n points and scale * *n triangles
  const int *n;
  int scale;
  __device__ void operator()(DState &d, int *) const {
    d.req_p = *n;
    d.req_t = scale * *n;
  }
};
struct RefreshedPoints {  // updateEmptyPoints done: the list holds lenp slots
  __device__ void operator()(DState &d, int *) const { d.nempty_p = d.lenp; }
};
struct RefreshedTris {
  __device__ void operator()(DState &d, int *) const { d.nempty_t = d.lent; }
};
struct GrowPoints {  // blocks of pointblock slots until the batch fits
  __device__ void operator()(DState &d, int *err) const {
    d.grew = 0;
    if (d.pointblock <= 0) {
      atomicCAS(err, 0, GQM_ERR_ARGUMENT);
      return;
    }
    long long num = 0;
    while (d.req_p > d.nempty_p + num * d.pointblock) num++;
    if (!num) return;
    const long long cap = d.pcap + num * d.pointblock;
    if (cap > d.pphys) {
      d.need_grow |= 1;
      return;
    }
    d.pcap = (int)cap;
    d.grew = 1;
  }
};
struct GrowTris {
  __device__ void operator()(DState &d, int *err) const {
    d.grew = 0;
    if (d.triblock <= 0) {
      atomicCAS(err, 0, GQM_ERR_ARGUMENT);
      return;
    }
    long long num = 0;
    while (d.req_t > d.nempty_t + num * d.triblock) num++;
    if (!num) return;
    const long long cap = d.tcap + num * d.triblock;
    if (cap > d.tphys) {
      d.need_grow |= 2;
      return;
    }
    d.tcap = (int)cap;
    d.grew = 1;
  }
};
struct SlotsReady {  // the batch's first free slots; no batch when the run must be repeated
  int *n;
  __device__ void operator()(DState &d, int *err) const {
    d.pslot = d.lenp - d.nempty_p;
    d.tslot = d.lent - d.nempty_t;
    if (!run_ok(d, err)) *n = 0;
  }
};
// slot bookkeeping after an insertion batch (refine.cu:3545-3559, 5354-5368)
struct ConsumeSlots {
  const int *n;
  int scale;
  __device__ void operator()(DState &d, int *) const {
    const int npts = *n, ntris = scale * *n;
    int slot_after = d.pcap - d.last_point;
    int slot_before = d.nempty_p - slot_after;
    if (slot_before < npts) d.last_point += npts - slot_before;
    d.nempty_p -= npts;
    slot_after = d.tcap - d.last_triangle;
    slot_before = d.nempty_t - slot_after;
    if (slot_before < ntris) d.last_triangle += ntris - slot_before;
    d.nempty_t -= ntris;
  }
};
struct SubsegRoom {  // the new subsegments of a midpoint batch fit
  __device__ void operator()(DState &d, int *) const {
    if (d.last_subseg + d.nenc > d.sphys) {
      d.need_grow |= 4;
      d.nenc = 0;
    }
  }
};
struct SubsegsAdded {
  __device__ void operator()(DState &d, int *) const { d.last_subseg += d.nenc; }
};
struct CavityRoom {  // the candidates' cavities fit their store
  __device__ void operator()(DState &d, int *) const {
    if (d.nbad > d.cav_cap) {
      d.need_grow |= 8;
      d.nbad = 0;
    }
  }
};
struct OuterReset {
  __device__ void operator()(DState &d, int *) const { d.outer = 0; }
};
struct RoundDone {
  __device__ void operator()(DState &d, int *) const { d.rounds++; }
};

// fills whose count (and offset) an earlier kernel wrote
__global__ void k_fill_n(int *a, DevInt n, int v) {
  const int cnt = nval(n);
  GS_LOOP(i, cnt) a[i] = v;
}
__global__ void k_fill_at(int *base, DevInt off, DevInt n, int v) {
  int *a = base + nval(off);
  const int cnt = nval(n);
  GS_LOOP(i, cnt) a[i] = v;
}

// Ordered compaction over [0, *hi) whose bound an earlier kernel wrote, in one
// launch of kDevCompactBlocks blocks: each block takes the next chunk (whole
// tiles) in the order the blocks start (a claimed counter, so every chunk
// before a block's own belongs to a block that is already running), counts
// it, publishes the count, adds up its predecessors' published values back to
// the nearest full prefix (decoupled look-back, 32 predecessors at a time),
// publishes its own prefix and emits.  Chunks past the end of the range are
// skipped (a short range is one block's work, with no look-back), the block
// of the last chunk writes the total, and the last block to finish clears the
// published words and the counters for the next call.  Every wait is
// bounded: a wait that runs out records GQM_ERR_TOPOLOGY and the block goes on.
constexpr int kDevCompactBlocks = 296;
constexpr long long kLookbackSpins = 1ll << 22;
struct CompactSync {
  unsigned long long word[kDevCompactBlocks];  // (state << 32) | value; state 1: count, 2: prefix through the chunk
  unsigned next_chunk, finished;
};
__device__ __forceinline__ int dev_chunk(int n) {
  int chunk = (n + kDevCompactBlocks - 1) / kDevCompactBlocks;
  chunk = max(chunk, kCompactTile);
  return (chunk + kCompactTile - 1) / kCompactTile * kCompactTile;
}
template <class F, class Mp>
__global__ void __launch_bounds__(kCompactThreads) k_compact1(F f, Mp m, DevInt hi_, int *out, int *total,
                                                              CompactSync *cs, int *err) {
  __shared__ int wsum[kCompactThreads / 32];
  __shared__ int sh_chunk, sh_base;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) sh_chunk = (int)atomicAdd(&cs->next_chunk, 1u);
  __syncthreads();
  const int b = sh_chunk;
  const int hi = nval(hi_), chunk = dev_chunk(hi);
  const int last = hi > 0 ? (hi - 1) / chunk : 0;  // the last chunk with elements (0 for an empty range)
  if (b <= last) {  // (the same for the whole block)
    const int b0 = min(hi, b * chunk), b1 = min(hi, b0 + chunk);
    // count
    int c = 0;
    for (int s = b0 + threadIdx.x * kCompactItems; s < b1; s += kCompactTile) {
#pragma unroll
      for (int j = 0; j < kCompactItems; ++j)
        if (s + j < b1 && f(s + j)) ++c;
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if (lane == 0) wsum[warp] = c;
    __syncthreads();
    if (warp == 0) {  // publish, then look back 32 predecessors at a time
      int cnt = 0;
      for (int w = 0; w < kCompactThreads / 32; ++w) cnt += wsum[w];
      volatile unsigned long long *word = cs->word;
      int prefix = 0;
      if (b == 0) {
        if (lane == 0) atomicExch(&cs->word[0], (2ull << 32) | (unsigned)cnt);
      } else {
        if (lane == 0) atomicExch(&cs->word[b], (1ull << 32) | (unsigned)cnt);
        for (int top = b - 1; top >= 0; top -= 32) {
          const int j = top - lane;
          unsigned long long v = 2ull << 32;  // before chunk 0: a prefix of zero
          if (j >= 0) {
            v = word[j];
            long long spins = 0;
            while ((v >> 32) == 0 && ++spins < kLookbackSpins) v = word[j];
            if ((v >> 32) == 0) {  // gave up: the count is wrong, and the run reports it
              atomicCAS(err, 0, GQM_ERR_TOPOLOGY);
              v = 2ull << 32;
            }
          }
          const unsigned full = __ballot_sync(0xffffffffu, (v >> 32) == 2);
          const int stop = full ? __ffs(full) - 1 : 31;  // the nearest full prefix (lane 0 is the nearest chunk)
          int x = lane <= stop ? (int)(unsigned)v : 0;
          for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
          prefix += __shfl_sync(0xffffffffu, x, 0);
          if (full) break;
        }
        if (lane == 0) atomicExch(&cs->word[b], (2ull << 32) | (unsigned)(prefix + cnt));
      }
      if (lane == 0) {
        sh_base = prefix;
        if (b == last) *total = prefix + cnt;
      }
    }
    __syncthreads();
    // emit
    int base = sh_base;
    for (int tile = b0; tile < b1; tile += kCompactTile) {
      const int s = tile + threadIdx.x * kCompactItems;
      unsigned bits = 0;
#pragma unroll
      for (int j = 0; j < kCompactItems; ++j)
        if (s + j < b1 && f(s + j)) bits |= 1u << j;
      const int cc = __popc(bits);
      int x = cc;
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
      }
      if (lane == 31) wsum[warp] = x;
      __syncthreads();
      int woff = 0, tot = 0;
#pragma unroll
      for (int w = 0; w < kCompactThreads / 32; ++w) {
        const int v = wsum[w];
        woff += (w < warp) ? v : 0;
        tot += v;
      }
      int pos = base + woff + x - cc;
      while (bits) {
        const int j = __ffs(bits) - 1;
        bits &= bits - 1;
        out[pos++] = m(s + j);
      }
      base += tot;
      __syncthreads();
    }
  }
  // the last block to finish: a clean slate for the next call
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(&cs->finished, 1u) == kDevCompactBlocks - 1) {
      __threadfence();
      for (int j = 0; j <= last; ++j) cs->word[j] = 0;
      cs->next_chunk = 0;
      cs->finished = 0;
      __threadfence();
    }
  }
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
  int pointblock = 0, triblock = 0;
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
  // the driver's state on the device, and the refinement captured as one
  // CUDA graph (loops and branches as conditional nodes)
  DState *ds = nullptr;
  CompactSync *csync = nullptr;  // look-back words of the one-launch compactions (zero between calls)
  DState hds{};             // host copy: written before a run, read after it
  bool use_graph = true;    // false: the host reads each condition (GQM_NO_GRAPH=1, emulated build)
  bool capturing = false;   // the refinement graph is being captured
  cudaGraph_t ref_graph = nullptr;
  cudaGraphExec_t ref_exec = nullptr;
  long buf_gen = 0;         // bumped whenever a device buffer is allocated again
  int node_count = 0, cur_node = 0, node_id = 0;
  long long node_kernels[kMaxNodes + 1] = {};  // kernels in each conditional node's body; [kMaxNodes]: top level
  // physical capacities that a repeated run asks for (a run that would exceed
  // one stops and is repeated with larger buffers)
  long want_p = 0, want_t = 0, want_s = 0, want_cav = 0;
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
  // exploration run for descendant-count labels (gqm_learn_explore): the
  // rows' device arrays, and per-slot lineage sized with the mesh buffers at
  // the start of every attempt (a run is host-driven while exploring)
  bool explore = false;
  ExploreDev ex{};
  size_t ex_vrow_n = 0, ex_crow_n = 0, ex_mlin_n = 0;
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

  void release() {
    drop_ref_graph();
    void *ptrs[] = {M.pts, M.ps, M.pred, M.tv, M.tn, M.tsg, M.tst, M.tflip, M.tfo, M.flip0, M.tmark, M.tpos,
                    M.s2t, M.s2seg, M.enc, M.err, stm, emptyt, bad, imark, ilist, sinks, wl, act, win, neg, ll, sl,
                    newidx, tail, center, emptyp, pnew, enclist, encl2, smark, mids, snap, segs, dcount, bc,
                    dctr, dgc, dinput, mlp_w, mlp_b, M.fstamp, M.tstamp, fq, tl, clr, fc, cav, cavn, ktm, M.wbits, M.wcnt, M.wsup, M.wmeg,
                    ds, csync};
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
    ds = nullptr;
    csync = nullptr;
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
    for (void *q : {(void *)ex.vrow, (void *)ex.crow, (void *)ex.mlin})
      if (q) cudaFree(q);
    ex.vrow = ex.crow = ex.mlin = nullptr;
    ex_vrow_n = ex_crow_n = ex_mlin_n = 0;
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
          dalloc(&M.err, 1) || dalloc(&fc, 1) || dalloc(&ktm, 1) || dalloc(&stm, 1) || dalloc(&ds, 1) ||
          dalloc(&csync, 1))
        return GQM_ERR_MEMORY;
      cudaMemsetAsync(csync, 0, sizeof(CompactSync), st);
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
    count_launch(1);                             \
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
    buf_gen++;
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
    buf_gen++;
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
    buf_gen++;
    return GQM_OK;
  }

  // ==========================================================================
  // Control flow of the driver.  Every count and every piece of the
  // reference's slot bookkeeping lives in DState on the device.  While the
  // refinement graph is captured (capturing), a loop or a branch becomes a
  // conditional node of the graph whose condition a one-thread kernel sets on
  // the device; otherwise (the emulated build, GQM_NO_GRAPH=1) the same kernel
  // writes the condition to ds->flag and the host reads it.  Either way the
  // device runs the same kernels in the same order.
  // ==========================================================================
  static constexpr int kDevGrid = 148 * 8;  // grid of the kernels whose count is read on the device
#define DLAUNCH(kernel, ...)                  \
  do {                                        \
    KL(kernel, kDevGrid, 256)(__VA_ARGS__);   \
    count_launch(1);                          \
  } while (0)
#define DSTEP(f)                               \
  do {                                         \
    KL(k_do, 1, 32)(f, ds, M.err);             \
    count_launch(1);                           \
  } while (0)
  void count_launch(int n) {
    if (capturing)
      node_kernels[cur_node]++;
    else
      stats.kernel_launches += n;
  }
  int read_word(const int *dword, int *v) {
    cudaMemcpyAsync(hcount + C_MISC, dword, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return GQM_ERR_CUDA;
    stats.host_syncs++;
    *v = hcount[C_MISC];
    return GQM_OK;
  }
  // A loop (WHILE) or branch (IF).  pre(h, graph) launches the kernel that sets
  // the first condition, body(h, graph) the body's kernels; flag is the word
  // the condition kernels write.  For a loop, the body ends by setting the
  // next condition: itself (body_sets_cond) or with pre's kernel again.
  template <class Pre, class Body>
  int cond_node(bool loop, Pre pre, Body body, const int *flag, bool body_sets_cond) {
    cudaGraphConditionalHandle h{};
    if (!capturing) {
      pre(h, 0);
      for (;;) {
        int v = 0;
        int rc = read_word(flag, &v);
        if (rc || !v) return rc;
        rc = body(h, 0);
        if (rc || !loop) return rc;
        if (!body_sets_cond) pre(h, 0);
      }
    }
#ifdef GQM_HOST_EMU
    return GQM_ERR_CUDA;
#else
    if (node_count >= kMaxNodes) return GQM_ERR_CUDA;
    const int id = node_count++;
    cudaStreamCaptureStatus cs;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t nd = 0;
    if (cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &nd) != cudaSuccess ||
        cs != cudaStreamCaptureStatusActive)
      return GQM_ERR_CUDA;
    if (cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault) != cudaSuccess) return GQM_ERR_CUDA;
    node_id = id;
    pre(h, 1);
    if (cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &nd) != cudaSuccess) return GQM_ERR_CUDA;
    std::vector<cudaGraphNode_t> dv(deps, deps + nd);
    cudaGraph_t ended = nullptr;
    if (cudaStreamEndCapture(st, &ended) != cudaSuccess) return GQM_ERR_CUDA;
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = loop ? cudaGraphCondTypeWhile : cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    cudaGraphNode_t node = nullptr;
    if (cudaGraphAddNode(&node, g, dv.data(), dv.size(), &cp) != cudaSuccess) return GQM_ERR_CUDA;
    if (cudaStreamBeginCaptureToGraph(st, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal) != cudaSuccess)
      return GQM_ERR_CUDA;
    const int outer = cur_node;
    cur_node = id;
    int rc = body(h, 1);
    if (rc == 0 && loop && !body_sets_cond) {
      node_id = id;
      pre(h, 1);
    }
    cur_node = outer;
    cudaGraph_t bg = nullptr;
    if (cudaStreamEndCapture(st, &bg) != cudaSuccess && rc == 0) rc = GQM_ERR_CUDA;
    if (rc) return rc;
    if (cudaStreamBeginCaptureToGraph(st, g, &node, nullptr, 1, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
      return GQM_ERR_CUDA;
    return GQM_OK;
#endif
  }
  // a loop or branch on a DState condition functor
  template <class C, class Body>
  int dev_while(C c, Body body) {
    return cond_node(
        true,
        [&](cudaGraphConditionalHandle h, int graph) {
          KL(k_cond, 1, 32)(c, ds, M.err, h, graph, graph ? node_id : kMaxNodes);
          count_launch(1);
        },
        [&](cudaGraphConditionalHandle, int) { return body(); }, &ds->flag, false);
  }
  template <class C, class Body>
  int dev_if(C c, Body body) {
    return cond_node(
        false,
        [&](cudaGraphConditionalHandle h, int graph) {
          KL(k_cond, 1, 32)(c, ds, M.err, h, graph, graph ? node_id : kMaxNodes);
          count_launch(1);
        },
        [&](cudaGraphConditionalHandle, int) { return body(); }, &ds->flag, false);
  }
  // ordered compaction over [0, *hi) into out, count into *cnt
  template <class F, class Mp>
  void compact_dev(F f, Mp m, const int *hi, int *out, int *cnt) {
#ifdef GQM_HOST_EMU
    int c = 0;
    for (int i = 0; i < *hi; ++i)
      if (f(i)) out[c++] = m(i);
    *cnt = c;
    count_launch(1);
#else
    KL(k_compact1, kDevCompactBlocks, kCompactThreads)(f, m, DevInt{hi}, out, cnt, csync, M.err);
    count_launch(1);
#endif
  }

  // ---- free-slot bookkeeping (refine.cu:149-197, 3408-3444, 5259-5296) ----
  // updateEmptyPoints / updateEmptyTriangles
  void refresh_points() {
    compact_dev(PPtDeleted{M.ps}, Ident{}, &ds->pcap, emptyp, &ds->lenp);
    DSTEP(RefreshedPoints{});
  }
  void refresh_tris() {
    compact_dev(PTriNull{M.tst}, Ident{}, &ds->tcap, emptyt, &ds->lent);
    DSTEP(RefreshedTris{});
  }
  // room for *n points and scale * *n triangles; *n becomes 0 when the run
  // has to be repeated with larger buffers
  int ensure_slots(int *n, int scale) {
    DSTEP((SlotsRequest{n, scale}));
    int rc = dev_if(CondNeedPoints{}, [&] {
      refresh_points();
      DSTEP(GrowPoints{});
      return dev_if(CondGrew{}, [&] {
        refresh_points();
        return GQM_OK;
      });
    });
    if (rc) return rc;
    rc = dev_if(CondNeedTris{}, [&] {
      refresh_tris();
      DSTEP(GrowTris{});
      return dev_if(CondGrew{}, [&] {
        refresh_tris();
        return GQM_OK;
      });
    });
    if (rc) return rc;
    DSTEP(SlotsReady{n});
    return GQM_OK;
  }
  DevSlots pslots() const { return DevSlots{emptyp, &ds->pslot}; }
  DevSlots tslots() const { return DevSlots{emptyt, &ds->tslot}; }

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
  } tune;
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

  // ---- flip-flop (refine.cu:2328-2490) over the triangles flagged below last_triangle ----
  int flip_flop() {
    NvtxRange nvtx("gqm:flip_flop");
    DLAUNCH(k_flip_entry_reset, M, DevInt{&ds->last_triangle});
    compact_dev(PNotNullFlag{M.tst, M.tflip}, Ident{}, &ds->last_triangle, act, &fc->nact);
    return cond_node(
        true,
        [&](cudaGraphConditionalHandle h, int graph) {
          KL(k_flip_prep, 1, 32)(fc, h, graph);
          count_launch(1);
        },
        [&](cudaGraphConditionalHandle h, int graph) {
          flip_body(h, graph);
          // in a graph the steps are counted after the run (FlipCtl::steps)
          if (!capturing) stats.kernel_launches += step_kernels();
          return GQM_OK;
        },
        &fc->cond, true);
  }

  // ---- splitEncsegs (refine.cu:3180-3778) ----
  int split_encsegs() {
    NvtxRange nvtx("gqm:split_encsegs");
    DSTEP(OuterReset{});
    compact_dev(PNonNeg{M.enc}, Ident{}, &ds->last_subseg, enclist, &ds->nenc);
    return dev_while(CondEncroached{}, [&] {
      // delete free Steiner points inside diametral circles
      DLAUNCH(k_copy, smark, enclist, &ds->nenc);
      compact_dev(PNonNeg{smark}, ValueOf{smark}, &ds->nmark, mids, &ds->ndel);
      int rc = dev_while(CondDelete{}, [&] {
        DLAUNCH(k_mark_redundant, M, smark, mids, &ds->ndel);
        int r = flip_flop();
        if (r) return r;
        compact_dev(PNonNeg{smark}, ValueOf{smark}, &ds->nmark, mids, &ds->ndel);
        return GQM_OK;
      });
      if (rc) return rc;
      // insert the midpoints of the encroached subsegments
      rc = ensure_slots(&ds->nenc, 2);
      if (rc) return rc;
      DSTEP(SubsegRoom{});
      DLAUNCH(k_fill_at, M.enc, DevInt{&ds->last_subseg}, DevInt{&ds->nenc}, -1);
      DLAUNCH(k_copy, smark, enclist, &ds->nenc);
      compact_dev(PNonNeg{smark}, Ident{}, &ds->nenc, mids, &ds->nmid);
      rc = dev_while(CondMidpoints{}, [&] {
        DLAUNCH(k_reset_mid, M, mids, &ds->nmid, smark);
        DLAUNCH(k_mark_mid, M, mids, &ds->nmid, smark);
        DLAUNCH(k_mid_snapshot, M, mids, &ds->nmid, smark, snap);
        if (explore) DLAUNCH(k_explore_mid_pre, M, &ds->nmid, snap, ex);
        KL(k_bump_epoch, 1, 32)(fc);
        count_launch(1);
        DLAUNCH(k_insert_mid, M, mids, &ds->nmid, smark, snap, pslots(), tslots(), DevInt{&ds->last_subseg},
                &fc->epoch, dctr + 1);
        if (explore) DLAUNCH(k_explore_mid_post, M, mids, &ds->nmid, pslots(), ex);
        DLAUNCH(k_update_mid_nbrs, M, mids, &ds->nmid, smark, enclist);
        compact_dev(PNonNeg{smark}, Ident{}, &ds->nenc, mids, &ds->nmid);
        return GQM_OK;
      });
      if (rc) return rc;
      DSTEP((ConsumeSlots{&ds->nenc, 2}));
      DSTEP(SubsegsAdded{});
      rc = flip_flop();
      if (rc) return rc;
      compact_dev(PNonNeg{M.enc}, Ident{}, &ds->last_subseg, enclist, &ds->nenc);
      return GQM_OK;
    });
  }

  // ---- splitTriangles (refine.cu:5107-5547) on the ds->nbad triangles in `bad` ----
  int split_triangles() {
    NvtxRange nvtx("gqm:split_triangles");
    const int *dn = &ds->nbad;
    DSTEP(CavityRoom{});
    DLAUNCH(k_copy, imark, bad, dn);
    DLAUNCH(k_copy, ilist, bad, dn);
    DLAUNCH(k_circumcenter, M, bad, dn, (double)offconstant, offcenter, center);
    if (col_feat) DLAUNCH(k_collect, M, bad, dn, center, col_feat, col_tgt, col_cnt, col_cap);
    if (explore) DLAUNCH(k_explore_place, M, bad, dn, center, ex);
    if (placement == GQM_PLACE_LEARNED) {  // eight warps of a block take 256 candidates per pass
      KL(k_learned_place, kDevGrid, 32 * kInferWarpsMax)(M, bad, dn, mlp_dev(mlp_w, mlp_b), center, dctr + 4);
      count_launch(1);
    }
    DLAUNCH(k_fill_n, M.tmark, DevInt{&ds->last_triangle}, kMaxInt);
    if (pred_mode)
      DLAUNCH(k_locate<1>, M, bad, dn, center, sinks);
    else
      DLAUNCH(k_locate<0>, M, bad, dn, center, sinks);
    DLAUNCH(k_remove_losers, M, bad, dn, sinks, imark);
    DLAUNCH(k_fill_n, M.tmark, DevInt{&ds->last_triangle}, kMaxInt);
    // stored cavities: kCavityCap rows of cav_cap entries
    if (pred_mode)
      DLAUNCH(k_cavity_mark<1>, M, dn, sinks, center, imark, ilist, cav, cavn, (int)cav_cap);
    else
      DLAUNCH(k_cavity_mark<0>, M, dn, sinks, center, imark, ilist, cav, cavn, (int)cav_cap);
    DLAUNCH(k_cavity_check, M, dn, cav, cavn, (int)cav_cap, imark, ilist);
    compact_dev(PNonNeg{imark}, Ident{}, dn, wl, &ds->nst);
    DLAUNCH(k_fill_n, encl2, DevInt{&ds->last_subseg}, -1);
    DLAUNCH(k_mark_onsegs, M, wl, &ds->nst, sinks, encl2);
    int rc = ensure_slots(&ds->nst, 2);
    if (rc) return rc;
    DLAUNCH(k_reset_steiner, M, wl, &ds->nst, sinks);
    KL(k_bump_epoch, 1, 32)(fc);
    count_launch(1);
    DLAUNCH(k_insert_steiner, M, wl, &ds->nst, sinks, center, pslots(), tslots(), &fc->epoch, dctr + 0);
    if (explore) DLAUNCH(k_explore_steiner, M, wl, &ds->nst, center, pslots(), ex);
    DLAUNCH(k_update_steiner_nbrs, M, wl, &ds->nst, sinks);
    DSTEP((ConsumeSlots{&ds->nst, 2}));
    rc = flip_flop();
    if (rc) return rc;
    DLAUNCH(k_onsegs_to_enc, M, encl2, DevInt{&ds->last_subseg});
    return GQM_OK;
  }

  // ---- the refinement proper (refine.cu:6830-7024), from the initialised mesh ----
  // the network's device copy (bf16 weights, fp32 biases)
  int set_network(const float *params) {
    if (!mlp_w && (dalloc(&mlp_w, kMlpW) || dalloc(&mlp_b, kMlpB))) return GQM_ERR_MEMORY;
    std::vector<uint16_t> hw(kMlpW);
    std::vector<float> hb(kMlpB);
    mlp_pack(params, hw.data(), hb.data());
    cudaMemcpyAsync(mlp_w, hw.data(), sizeof(uint16_t) * kMlpW, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(mlp_b, hb.data(), sizeof(float) * kMlpB, cudaMemcpyHostToDevice, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return GQM_ERR_CUDA;
    return GQM_OK;
  }
  // lineage arrays sized with this attempt's buffers, rows counted from zero
  int explore_begin() {
    if (grow_dev(&ex.vrow, &ex_vrow_n, (size_t)pphys) || grow_dev(&ex.crow, &ex_crow_n, (size_t)tphys) ||
        grow_dev(&ex.mlin, &ex_mlin_n, (size_t)std::max<long>(sphys, 1)))
      return GQM_ERR_MEMORY;
    cudaMemsetAsync(ex.vrow, 0xff, sizeof(int) * (size_t)pphys, st);
    cudaMemsetAsync(ex.cnt, 0, sizeof(unsigned long long), st);
    return GQM_OK;
  }
  int refine_body() {
    if (explore) {
      if (capturing) return GQM_ERR_ARGUMENT;  // exploration runs are host-driven
      int rc = explore_begin();
      if (rc) return rc;
    }
    refresh_points();
    refresh_tris();
    DLAUNCH(k_mark_all_encsegs, M, DevInt{&ds->last_subseg});  // last_subseg = the input's subsegments here
    int rc = split_encsegs();
    if (rc) return rc;
    DLAUNCH(k_mark_bad, M, DevInt{&ds->last_triangle});
    compact_dev(PBad{M.tst}, Ident{}, &ds->last_triangle, bad, &ds->nbad);
    return dev_while(CondRound{}, [&] {
      int r = split_triangles();
      if (r) return r;
      r = split_encsegs();
      if (r) return r;
      DLAUNCH(k_points_old, M, DevInt{&ds->last_point});
      DSTEP(RoundDone{});
      DLAUNCH(k_mark_bad, M, DevInt{&ds->last_triangle});
      compact_dev(PBad{M.tst}, Ident{}, &ds->last_triangle, bad, &ds->nbad);
      return GQM_OK;
    });
  }

  // Everything the captured refinement graph depends on besides DState: a
  // change in any of it captures the graph again.
  struct RefKey {
    Mesh M;
    long buf_gen;
    int pred_mode, placement, offcenter, offconstant;
    const void *col_feat, *col_tgt, *col_cnt, *mlp_w, *mlp_b;
    unsigned long long col_cap;
    Tuning tune;
  };
  RefKey ref_key{};  // what the captured graph was built for
  RefKey ref_key_now() const {
    RefKey k;
    memset(&k, 0, sizeof(k));
    k.M = M;
    k.buf_gen = buf_gen;
    k.pred_mode = pred_mode;
    k.placement = placement;
    k.offcenter = offcenter;
    k.offconstant = offconstant;
    k.col_feat = col_feat;
    k.col_tgt = col_tgt;
    k.col_cnt = col_cnt;
    k.mlp_w = mlp_w;
    k.mlp_b = mlp_b;
    k.col_cap = col_cap;
    k.tune = tune;
    return k;
  }
  void drop_ref_graph() {
#ifndef GQM_HOST_EMU
    if (ref_exec) cudaGraphExecDestroy(ref_exec);
    if (ref_graph) cudaGraphDestroy(ref_graph);
#endif
    ref_exec = nullptr;
    ref_graph = nullptr;
  }
  int capture_refinement() {
#ifdef GQM_HOST_EMU
    return GQM_ERR_CUDA;
#else
    drop_ref_graph();
    node_count = 0;
    cur_node = kMaxNodes;
    memset(node_kernels, 0, sizeof(node_kernels));
    cudaGraph_t g = nullptr;
    if (cudaGraphCreate(&g, 0) != cudaSuccess) return GQM_ERR_CUDA;
    if (cudaStreamBeginCaptureToGraph(st, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      cudaGraphDestroy(g);
      return GQM_ERR_CUDA;
    }
    capturing = true;
    const long long launches = stats.kernel_launches;
    int rc = refine_body();
    capturing = false;
    stats.kernel_launches = launches;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(st, &cs);
    if (cs != cudaStreamCaptureStatusNone) {
      cudaGraph_t t = nullptr;
      if (cudaStreamEndCapture(st, &t) != cudaSuccess && rc == 0) rc = GQM_ERR_CUDA;
    }
    if (rc == 0 && cudaGraphInstantiate(&ref_exec, g, 0) != cudaSuccess) {
      ref_exec = nullptr;
      rc = GQM_ERR_CUDA;
    }
    if (rc) {
      cudaGraphDestroy(g);
      cudaGetLastError();
      return rc;
    }
    ref_graph = g;
    ref_key = ref_key_now();
    return GQM_OK;
#endif
  }
  // one refinement from the initialised mesh: the captured graph (captured
  // again when what it depends on changed), or the same steps driven from the
  // host
  int run_refinement() {
    if (use_graph) {
      const RefKey k = ref_key_now();
      if (!ref_exec || memcmp(&k, &ref_key, sizeof(k)) != 0) {
        if (capture_refinement() != GQM_OK) use_graph = false;  // the host-driven steps below
      }
      if (use_graph) {
        if (cudaGraphLaunch(ref_exec, st) != cudaSuccess) return GQM_ERR_CUDA;
        stats.kernel_launches += node_kernels[kMaxNodes];
        return GQM_OK;
      }
    }
    return refine_body();
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
      int rc = set_network(opt->mlp);
      if (rc) return rc;
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
    want_p = want_t = want_s = want_cav = 0;
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
      // the caller's arrays are packed into pinned memory on the host's cores
      // and uploaded in pieces of 32 MB, the front while the back is packed
      if (grow_pinned(need)) return GQM_ERR_MEMORY;
      const size_t bp = sizeof(double) * 2 * np, bt = sizeof(int) * 3 * nt, bs = sizeof(int) * 2 * ns;
      const HostCopy parts[4] = {{h_stage, in->pointlist, bp}, {h_stage + bp, in->trianglelist, bt},
                                 {h_stage + bp + bt, in->neighborlist, bt},
                                 {h_stage + bp + 2 * bt, in->segmentlist, bs}};
      host_copy_streamed(parts, h_stage, 32u << 20, [&](size_t off, size_t bytes) {
        cudaMemcpyAsync(base + off, h_stage + off, bytes, cudaMemcpyHostToDevice, st);
      });
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
    int attempt = 0;
  restart:
    // physical buffers (logical capacities are tracked in DState)
#ifdef GQM_TEST_TIGHT_BUFFERS
    // test builds: physical buffers exactly the logical capacity, so a run
    // that grows the logical capacity is repeated with larger buffers
    rc = alloc_points(std::max<long>(std::max<long>(pcap, pphys), want_p));
    if (rc) return rc;
    rc = alloc_tris(std::max<long>(std::max<long>(tcap, tphys), want_t));
    if (rc) return rc;
#else
    rc = alloc_points(std::max<long>(std::max<long>(pcap + 3L * pointblock, pphys), want_p));
    if (rc) return rc;
    rc = alloc_tris(std::max<long>(std::max<long>(tcap + 4L * triblock, tphys), want_t));
    if (rc) return rc;
#endif
    rc = alloc_subsegs(std::max<long>(std::max<long>(4L * ns + 1024, sphys), want_s));
    if (rc) return rc;
    {  // stored cavities of the Steiner candidates: kCavityCap rows of cav_cap entries
      const long want = std::max<long>(std::max<long>(tcap / 4, 1024), want_cav);
      if (cav_cap < want) {
        if (cav) cudaFree(cav);
        if (cavn) cudaFree(cavn);
        cav = cavn = nullptr;
        cav_cap = 0;
        if (dalloc(&cav, (size_t)kCavityCap * want) || dalloc(&cavn, want)) return GQM_ERR_MEMORY;
        cav_cap = want;
        buf_gen++;
      }
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
    // the driver's state on the device: the reference's logical capacities
    // and high-water marks, and the physical capacities a run must stay in
    hds = DState{};
    hds.pcap = (int)pcap;
    hds.tcap = (int)tcap;
    hds.pphys = (int)pphys;
    hds.tphys = (int)tphys;
    hds.sphys = (int)sphys;
    hds.cav_cap = (int)cav_cap;
    hds.last_point = np;
    hds.last_triangle = nt;
    hds.last_subseg = ns;
    hds.pointblock = pointblock;
    hds.triblock = triblock;
    hds.max_rounds = max_rounds;
    cudaMemcpyAsync(ds, &hds, sizeof(DState), cudaMemcpyHostToDevice, st);
    rc = run_refinement();
    if (rc == 0) {
      cudaMemcpyAsync(&hds, ds, sizeof(DState), cudaMemcpyDeviceToHost, st);
      if (cudaStreamSynchronize(st) != cudaSuccess) rc = GQM_ERR_CUDA;
      stats.host_syncs++;
    }
    if (rc == 0 && hds.need_grow) {
      // a physical capacity would have been exceeded: repeat the run with
      // larger buffers (the result does not depend on them)
      if (++attempt > 8) return GQM_ERR_MEMORY;
      if (hds.need_grow & 1) want_p = 2 * pphys;
      if (hds.need_grow & 2) want_t = 2 * tphys;
      if (hds.need_grow & 4) want_s = 2 * sphys;
      if (hds.need_grow & 8) want_cav = 2 * cav_cap;
      pcap = np + pointblock;
      tcap = nt + triblock;
      stats = gqm_stats{};
      goto restart;
    }
    last_point = hds.last_point;
    last_triangle = hds.last_triangle;
    last_subseg = hds.last_subseg;
    pcap = hds.pcap;
    tcap = hds.tcap;
    stats.rounds = (int)hds.rounds;
    stats.bad_total = hds.bad_total;
    if (use_graph)  // kernels of the conditional nodes' bodies, times the bodies ran
      for (int i = 0; i < node_count; ++i) stats.kernel_launches += hds.iters[i] * node_kernels[i];
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
    unsigned long long hc[8];
    cudaMemcpy(hc, dctr, sizeof(hc), cudaMemcpyDeviceToHost);
    stats.learned_candidates = (long long)hc[4];
    stats.learned_used = (long long)hc[5];
    FlipCtl hf;
    cudaMemcpy(&hf, fc, sizeof(hf), cudaMemcpyDeviceToHost);
    stats.flip_steps = hf.steps;
    // with the graph, the kernels of every grid step of the flip-flop loops (a
    // grid step, its condition and the single-block kernel that runs the small
    // steps after it) are added here
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
    if (char *blk = pool_take(bytes)) {  // straight into a pinned block the caller owns until gqm_free_result
      cudaMemcpyAsync(blk, d_out, bytes, cudaMemcpyDeviceToHost, st);
      if (cudaStreamSynchronize(st) != cudaSuccess) {
        pool_give(blk);
        return GQM_ERR_CUDA;
      }
      out->numberofpoints = (int)np;
      out->numberoftriangles = (int)nt;
      out->numberofsegments = (int)ns;
      out->pointlist = (double *)blk;
      out->trianglelist = (int *)(blk + o_tri);
      out->neighborlist = (int *)(blk + o_nbr);
      out->segmentlist = (int *)(blk + o_seg);
      out->pstatus = (unsigned char *)(blk + o_ps);
      out->tstatus = (unsigned char *)(blk + o_ts);
      return GQM_OK;
    }
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
  // the device time of the flip-flop loops since this reset (FlipCtl)
  cudaMemsetAsync(&r.fc->loop_ns, 0, sizeof(r.fc->loop_ns), r.st);
  cudaMemsetAsync(&r.fc->loops, 0, sizeof(r.fc->loops), r.st);
  return cudaStreamSynchronize(r.st) == cudaSuccess ? GQM_OK : GQM_ERR_CUDA;
}
int gqm_context_probe_read(gqm_context *ctx, gqm_probe *p) {
  if (!ctx || !p || !ctx->r.ktm) return GQM_ERR_ARGUMENT;
  gqm::Refiner &r = ctx->r;
  if (cudaSetDevice(r.device) != cudaSuccess) return GQM_ERR_CUDA;
  gqm::KTimer h, hs;
  gqm::FlipCtl hf;
  if (cudaStreamSynchronize(r.st) != cudaSuccess ||
      cudaMemcpy(&h, r.ktm, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(&hs, r.stm, sizeof(hs), cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(&hf, r.fc, sizeof(hf), cudaMemcpyDeviceToHost) != cudaSuccess)
    return GQM_ERR_CUDA;
  p->small_launches = (long long)hs.launches;
  p->small_items = (long long)hs.items;
  p->small_winners = (long long)hs.winners;
  p->small_ms = (double)hs.total_ns * 1e-6;
  p->check_launches = (long long)h.launches;
  p->check_items = (long long)h.items;
  p->check_ms = (double)h.total_ns * 1e-6;
  for (int i = 0; i < 4; ++i) p->first_items[i] = (long long)h.first_items[i];
  p->loop_launches = (long long)hf.loops;
  p->loop_ms = (double)hf.loop_ns * 1e-6;
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
int gqm_learn_explore(const gqm_cdt_in *in, const gqm_options *opt, int levels, unsigned seed, const float *mlp,
                      float eps, float *features, int *level, float *t_used, int *parent, unsigned char *inserted,
                      int *midpoints, long long cap, long long *count) {
  if (!in || !opt || levels < 2 || levels > 64 || cap < 0 || cap > INT_MAX || !(eps >= 0.0f && eps <= 1.0f) ||
      (cap > 0 && (!features || !level || !t_used || !parent || !inserted || !midpoints)))
    return GQM_ERR_ARGUMENT;
  gqm_options o = *opt;
  o.placement = GQM_PLACE_PLAIN;  // the drawn points replace the off-centers
  o.mlp = nullptr;
  int rc = validate(in, &o);
  if (rc) return rc;
  gqm_context *ctx = nullptr;
  rc = gqm_context_create(o.device, &ctx);
  if (rc) return rc;
  gqm::Refiner &r = ctx->r;
  gqm::ExploreDev &E = r.ex;
  if (mlp && (rc = r.set_network(mlp)) != GQM_OK) {
    gqm_context_destroy(ctx);
    return rc;
  }
  E.use_net = mlp ? 1 : 0;
  E.eps = mlp ? eps : 1.0f;
  if (mlp) E.net = gqm::mlp_dev(r.mlp_w, r.mlp_b);
  const size_t rows = (size_t)(cap > 0 ? cap : 1);
  if (r.dalloc(&E.feat, rows * gqm::kFeat) || r.dalloc(&E.level, rows) || r.dalloc(&E.tused, rows) ||
      r.dalloc(&E.parent, rows) || r.dalloc(&E.ins, rows) || r.dalloc(&E.mids, rows) || r.dalloc(&E.cnt, 1)) {
    rc = GQM_ERR_MEMORY;
  } else {
    E.cap = (unsigned long long)cap;
    E.levels = levels;
    E.seed = seed;
    r.explore = true;
    r.use_graph = false;
    gqm_stats st;
    rc = gqm_context_run(ctx, in, 0, &o, &st);
    unsigned long long n = 0;
    if (!rc && cudaMemcpy(&n, E.cnt, sizeof(n), cudaMemcpyDeviceToHost) != cudaSuccess) rc = GQM_ERR_CUDA;
    if (count) *count = (long long)n;
    if (!rc && n > (unsigned long long)cap) rc = GQM_ERR_TOO_LARGE;  // lineage would be cut: no rows returned
    if (!rc && n > 0) {
      const size_t m = (size_t)n;
      if (cudaMemcpy(features, E.feat, sizeof(float) * gqm::kFeat * m, cudaMemcpyDeviceToHost) != cudaSuccess ||
          cudaMemcpy(level, E.level, sizeof(int) * m, cudaMemcpyDeviceToHost) != cudaSuccess ||
          cudaMemcpy(t_used, E.tused, sizeof(float) * m, cudaMemcpyDeviceToHost) != cudaSuccess ||
          cudaMemcpy(parent, E.parent, sizeof(int) * m, cudaMemcpyDeviceToHost) != cudaSuccess ||
          cudaMemcpy(inserted, E.ins, m, cudaMemcpyDeviceToHost) != cudaSuccess ||
          cudaMemcpy(midpoints, E.mids, sizeof(int) * m, cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = GQM_ERR_CUDA;
    }
  }
  for (void *q : {(void *)E.feat, (void *)E.level, (void *)E.tused, (void *)E.parent, (void *)E.ins, (void *)E.mids,
                  (void *)E.cnt})
    if (q) cudaFree(q);
  E.feat = nullptr;
  E.level = E.parent = E.mids = nullptr;
  E.tused = nullptr;
  E.ins = nullptr;
  E.cnt = nullptr;
  r.explore = false;
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
  if (gqm::pool_give(out->pointlist)) {  // one pinned block holds all six arrays
    memset(out, 0, sizeof(*out));
    return;
  }
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
