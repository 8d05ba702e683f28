// Device-side mesh layout and per-element helpers of the B200 refiner.
//
// Layout (structure of arrays, resident in HBM for the whole refinement):
//   pts   double2[Pcap]   vertex coordinates (one 128-bit load each)
//   ps    uint8[Pcap]     point flags: DELETED | STEINER | SEGSPLIT | NEW
//   pred  uint8[Pcap]     "redundant" flag (set concurrently by many threads)
//   tv    int4[Tcap]      triangle vertices (x, y, z), w unused
//   tn    int4[Tcap]      oriented neighbours (tri << 2 | edge), -1 boundary
//   tsg   int4[Tcap]      subsegment on each edge, -1 if none
//   tst   uint8[Tcap]     NOTNULL | BAD | CHECK
//   tflip uint8[Tcap]     flip-flop marker (set concurrently)
//   tfo   uint8[Tcap]     flip orientation code, 15 = none
//   tmark int[Tcap]       ownership marker (atomicMin) / flipBy
//   s2t   u128[Scap]      subsegment -> oriented triangle in the low word,
//                         tagged with the launch epoch and the storing
//                         thread's key (see s2t_store)
//   s2seg int[Scap], enc int[Scap], segs int2[S_in]
//   wbits uint32[Tcap/2^5], wcnt int[Tcap/2^10], wsup int[Tcap/2^15],
//   wmeg int[Tcap/2^20]   flip winners of a step (bitmap and counts)
// Edge i of a triangle joins vertices i+1 and i+2 and faces vertex i; an
// oriented triangle (t << 2 | i) names edge i of t (GPU_Refine/refine.cu:95-113).
// Flags the reference keeps in one byte (GPU_Refine/refine.h:36-205) are split
// across separate byte arrays so that concurrent writers never share a byte.
#pragma once
#include <cstdint>

#include "predicates.h"

namespace gqm {

constexpr int kMaxInt = 2147483647;
// subseg2tri entry: bits 127..64 launch epoch, 63..32 writer key, 31..0 oriented triangle
typedef unsigned __int128 s2t_t;
constexpr int kCavityCap = 50;  // MyList capacity, GPU_Refine/refine.h:30

enum : uint8_t { PS_DELETED = 1, PS_STEINER = 2, PS_SEGSPLIT = 4, PS_NEW = 8 };
enum : uint8_t { TS_NOTNULL = 1, TS_BAD = 2, TS_CHECK = 4 };

struct Mesh {
  double2 *pts;
  uint8_t *ps, *pred;
  int4 *tv, *tn, *tsg;
  uint8_t *tst, *tflip, *tfo, *flip0;
  int *tmark;
  int *tpos;  // winner-slot of each triangle during a flip step
  int *fstamp, *tstamp;  // per-triangle generation stamps deduplicating the flip-step queues
  s2t_t *s2t;
  // flip winners of the current step: one bit per triangle slot and winner
  // counts per 2^10, 2^15 and 2^20 slots (see win_rank)
  unsigned *wbits;
  int *wcnt, *wsup, *wmeg;
  int *s2seg, *enc;
  const int2 *segs;
  int *err;  // first error code raised on the device
  double gc2;  // cos^2(theta), computed on the device as the reference does
  double max_area;  // area bound (0: none): larger triangles are bad whatever their angles
  int mode;    // 1 Ruppert, 0 Chew
};

__device__ __forceinline__ int dtri(int o) { return o >= 0 ? (o >> 2) : -1; }
__device__ __forceinline__ int dori(int o) { return o & 3; }
__device__ __forceinline__ int etri(int t, int o) { return t >= 0 ? ((t << 2) | o) : -1; }
__device__ __forceinline__ int negate_idx(int i) { return -i - 3; }
__device__ __forceinline__ int m3(int i) { return i >= 3 ? i - 3 : i; }

__device__ __forceinline__ int comp(const int4 &v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }
__device__ __forceinline__ void setc(int4 &v, int i, int x) {
  if (i == 0)
    v.x = x;
  else if (i == 1)
    v.y = x;
  else
    v.z = x;
}
// single-component stores into an int4 row
__device__ __forceinline__ void st1(int4 *a, int t, int i, int x) { reinterpret_cast<int *>(a + t)[i] = x; }
__device__ __forceinline__ int ld1(const int4 *a, int t, int i) { return reinterpret_cast<const int *>(a + t)[i]; }

__device__ __forceinline__ int s2t_get(const Mesh &M, int s) { return (int)(uint32_t)M.s2t[s]; }
__device__ __forceinline__ s2t_t s2t_plain(int v) { return (s2t_t)(uint32_t)v; }  // epoch 0: older than any launch
// Key of a store into subseg2tri by the thread at position `pos` of a launch,
// `slot` being the store's place in the kernel's program order.  When threads
// of one launch store into the same entry, the largest key is kept: within a
// warp the later store instruction (a warp issues its stores in order) and,
// for one instruction, the lower lane; across warps the lower warp.  That is
// the order in which the reference's racing stores (GPU_Refine/refine.cu:
// 1362-1372, 1419-1424, 1533-1544, 2844-2850, 2900-2903, 4744-4876) were seen
// to land on a B200, and the oracle applies the same key.
__device__ __forceinline__ uint32_t wkey(int pos, int slot) {
  return ((0x7FFFFFu - ((uint32_t)pos >> 5)) << 9) | ((uint32_t)slot << 5) | (31u - ((uint32_t)pos & 31u));
}
// A value stored in an earlier launch always loses to one of this launch; in
// one launch the larger (epoch, key) wins.  The loop reads the entry with the
// compare-and-swap itself, so a torn read is never acted on.
__device__ __forceinline__ void s2t_store(const Mesh &M, int s, int v, uint32_t epoch, uint32_t key) {
  const s2t_t nw = ((s2t_t)epoch << 64) | ((s2t_t)key << 32) | (uint32_t)v;
  s2t_t cur = 0;
  for (;;) {
    const s2t_t o = atomicCAS(M.s2t + s, cur, nw);
    if (o == cur || (o >> 32) >= (nw >> 32)) return;
    cur = o;
  }
}

// Position of flip winner `index` in the reference's winner list, which is
// compacted in triangle order (kernelUpdatePhase1's pos, refine.cu:1312): the
// number of this step's winners with a smaller slot.  The winners' own list
// here is filled by atomics in any order, so the position is counted from the
// winner bitmap and its counts per 2^10, 2^15 and 2^20 slots: at most 31
// entries of each level (one 128-byte line each) plus the 2^20 counts before
// the slot, all independent loads.  Only stores into subseg2tri need it.
__device__ __forceinline__ int sum32(const int *a, int lo, int hi) {  // a[lo..hi), hi - lo < 32
  int r = 0;
#pragma unroll
  for (int j = 0; j < 31; ++j)
    if (lo + j < hi) r += a[lo + j];
  return r;
}
__device__ __forceinline__ int win_rank(const Mesh &M, int index) {
  const int w = index >> 5, c = index >> 10, sc = index >> 15, mg = index >> 20;
  int r = 0;
  for (int i = 0; i < mg; ++i) r += M.wmeg[i];
  r += sum32(M.wsup, mg << 5, sc) + sum32(M.wcnt, sc << 5, c);
  int b = 0;
#pragma unroll
  for (int j = 0; j < 31; ++j)
    if ((c << 5) + j < w) b += __popc(M.wbits[(c << 5) + j]);
  return r + b + __popc(M.wbits[w] & ((1u << (index & 31)) - 1u));
}
// Slot in a list whose length *n many threads bump at once: the lanes of a
// warp that arrive together take consecutive slots with one atomic, issued by
// the lowest of them, instead of one atomic each on the same word.  The order
// of the entries within a list is not used by any step.
__device__ __forceinline__ int list_slot(int *n) {
#ifdef GQM_HOST_EMU
  return atomicAdd(n, 1);
#else
  const unsigned m = __activemask();
  const int lane = (int)(threadIdx.x & 31u), leader = __ffs(m) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(n, __popc(m));
  base = __shfl_sync(m, base, leader);
  return base + __popc(m & ((1u << lane) - 1u));
#endif
}
// The same for an event counter: one atomic per warp.
__device__ __forceinline__ void count_event(unsigned long long *c) {
#ifdef GQM_HOST_EMU
  atomicAdd(c, 1ull);
#else
  const unsigned m = __activemask();
  if ((int)(threadIdx.x & 31u) == __ffs(m) - 1) atomicAdd(c, (unsigned long long)__popc(m));
#endif
}
// enter / leave the winner bitmap and its counts.  The two coarse counts
// (2^15 and 2^20 slots) are few and hot, so the lanes of a warp that hit the
// same one add together (one atomic per distinct counter); `on` says whether
// this lane takes part (every lane of the warp must call).
__device__ __forceinline__ void win_count(int *a, int idx, bool on, int d) {
#ifdef GQM_HOST_EMU
  if (on) atomicAdd(a + idx, d);
#else
  const unsigned act = __ballot_sync(0xffffffffu, on);
  if (!on) return;
  const unsigned same = __match_any_sync(act, idx);
  if ((int)(threadIdx.x & 31u) == __ffs(same) - 1) atomicAdd(a + idx, d * __popc(same));
#endif
}
__device__ __forceinline__ void win_mark(const Mesh &M, int index, bool on) {
  if (on) {
    atomicOr(M.wbits + (index >> 5), 1u << (index & 31));
    atomicAdd(M.wcnt + (index >> 10), 1);
  }
  win_count(M.wsup, on ? index >> 15 : -1, on, 1);
  win_count(M.wmeg, on ? index >> 20 : -1, on, 1);
}
__device__ __forceinline__ void win_unmark(const Mesh &M, int index, bool on) {
  if (on) {
    atomicAnd(M.wbits + (index >> 5), ~(1u << (index & 31)));
    atomicAdd(M.wcnt + (index >> 10), -1);
  }
  win_count(M.wsup, on ? index >> 15 : -1, on, -1);
  win_count(M.wmeg, on ? index >> 20 : -1, on, -1);
}

__device__ __forceinline__ void raise_err(const Mesh &M, int code) { atomicCAS(M.err, 0, code); }

// ---------------------------------------------------------------------------
// Predicates with the reference's effective arithmetic (PRED = 0) or exact
// (PRED = 1).  Orientation: cuda_fast / cuda_ccw.  Incircle: the
// "cuda_inCircle, then cuda_inCircle_exact if 0" pattern used by every caller.
// ---------------------------------------------------------------------------
template <int PRED>
__device__ __forceinline__ double orient(double2 a, double2 b, double2 c) {
  if (PRED == 0) return gqm_orient_ref(a.x, a.y, b.x, b.y, c.x, c.y);
  return gqm_orient_exact(a.x, a.y, b.x, b.y, c.x, c.y);
}
// Incircle tests that needed the expansion path (determinant exactly zero with
// the reference's arithmetic, filter inconclusive with exact arithmetic),
// summed over every refinement on the device since the last reset (one
// counter per compiled module).
static __device__ unsigned long long g_incircle_fallbacks;
template <int PRED>
__device__ __noinline__ double incircle_slow(double2 a, double2 b, double2 c, double2 d) {
  atomicAdd(&g_incircle_fallbacks, 1ull);
  if (PRED == 0) return gqm_incircle_zero_fallback_ref(a.x, a.y, b.x, b.y, c.x, c.y, d.x, d.y);
  return gqm_incircle_exact(a.x, a.y, b.x, b.y, c.x, c.y, d.x, d.y);
}
template <int PRED>
__device__ __forceinline__ double incircle(double2 a, double2 b, double2 c, double2 d) {
  if (PRED == 0) {
    double r = gqm_incircle_det_ref(a.x, a.y, b.x, b.y, c.x, c.y, d.x, d.y);
    if (r != 0) return r;
    return incircle_slow<0>(a, b, c, d);
  }
  // exact: filter then exact expansion
  double adx = a.x - d.x, bdx = b.x - d.x, cdx = c.x - d.x;
  double ady = a.y - d.y, bdy = b.y - d.y, cdy = c.y - d.y;
  double bdxcdy = bdx * cdy, cdxbdy = cdx * bdy, alift = adx * adx + ady * ady;
  double cdxady = cdx * ady, adxcdy = adx * cdy, blift = bdx * bdx + bdy * bdy;
  double adxbdy = adx * bdy, bdxady = bdx * ady, clift = cdx * cdx + cdy * cdy;
  double det = alift * (bdxcdy - cdxbdy) + blift * (cdxady - adxcdy) + clift * (adxbdy - bdxady);
  double perm = (fabs(bdxcdy) + fabs(cdxbdy)) * alift + (fabs(cdxady) + fabs(adxcdy)) * blift +
                (fabs(adxbdy) + fabs(bdxady)) * clift;
  double eb = (10.0 + 96.0 * GQM_EPS) * GQM_EPS * perm;
  if (det > eb || -det > eb) return det;
  return incircle_slow<1>(a, b, c, d);
}

// checkseg4encroach, GPU_Refine/refine.cu:115-139 (goodcoss squared once).
__device__ __forceinline__ bool encroached(double2 o, double2 d, double2 a, double gc2, int mode) {
  double dot = gqm_madd(o.x - a.x, d.x - a.x, (o.y - a.y) * (d.y - a.y));
  if (dot < 0.0) {
    if (mode || dot * dot >= (2.0 * gc2 - 1.0) * (2.0 * gc2 - 1.0) *
                                   gqm_madd(o.x - a.x, o.x - a.x, (o.y - a.y) * (o.y - a.y)) *
                                   gqm_madd(d.x - a.x, d.x - a.x, (d.y - a.y) * (d.y - a.y)))
      return true;
  }
  return false;
}

}  // namespace gqm
