// Batched refinement of many independent domains in one persistent launch.
//
// Each thread block is a complete refiner for one domain at a time: the
// driver of refine.cu (GPU_Refine_Quality's control flow,
// GPU_Refine/refine.cu:6500-7139, with its free-slot bookkeeping) runs on the
// device, every thread of the block executing the same scalar control flow,
// and every pipeline step is the same kernel source as the single-domain path
// (kernels.cuh compiled in CTA mode: the block's threads stride over the
// domain's items and __syncthreads() separates the steps).  Blocks take
// domains from a queue ordered largest first (one atomic counter), so the
// whole batch, including every domain's round loop and flip-flop loop, is
// decided on the device: no host round trip and no launch per step.
//
// A domain's result is the one the single-domain path returns for it: the
// same steps run in the same order on the same slot discipline.  Each block
// owns one scratch arena sized for the largest domain of the batch; a domain
// whose mesh would outgrow its arena stops with GQM_ERR_ARENA and is refined
// again by the single-domain path on the host side of the call.
#define GQM_CTA_MODE 1
#define gqm gqm_cta
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "host_copy.h"

#include "../../include/gqm_refine.h"
#include "kernels.cuh"

namespace gqm {

// ---------------------------------------------------------------------------
// Block-wide helpers (every thread of the block calls them)
// ---------------------------------------------------------------------------

// Ordered compaction: out[k] = map(i) for the k-th i in [lo, hi) with pred(i),
// ascending; returns the count (the same value in every thread).  scan holds
// 33 ints of shared memory.
template <class F, class Mp>
__device__ int cta_compact(F f, Mp m, int lo, int hi, int *out, int *scan) {
  const int lane = (int)(threadIdx.x & 31u), w = (int)(threadIdx.x >> 5);
  const int nw = (int)((blockDim.x + 31u) >> 5);
  int base = 0;
  for (int t0 = lo; t0 < hi; t0 += (int)blockDim.x) {
    const int i = t0 + (int)threadIdx.x;
    const bool p = i < hi && f(i);
    const unsigned b = __ballot_sync(0xffffffffu, p);
    if (lane == 0) scan[w] = __popc(b);
    __syncthreads();
    if (w == 0) {
      const int v = lane < nw ? scan[lane] : 0;
      int x = v;
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
      }
      scan[lane] = x - v;
      const int total = __shfl_sync(0xffffffffu, x, 31);
      if (lane == 0) scan[32] = total;
    }
    __syncthreads();
    if (p) out[base + scan[w] + __popc(b & ((1u << lane) - 1u))] = m(i);
    base += scan[32];
    __syncthreads();
  }
  return base;
}
template <class T>
__device__ __forceinline__ void cta_fill(T *a, long n, T v) {
  for (long i = threadIdx.x; i < n; i += blockDim.x) a[i] = v;
}
__device__ __forceinline__ void cta_copy(int *dst, const int *src, int n) {
  for (int i = (int)threadIdx.x; i < n; i += (int)blockDim.x) dst[i] = src[i];
}
#define SYNC() __syncthreads()

// predicates and maps of the compactions (the same as refine.cu's)
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

// launch timer that is never on (the block path is timed as a whole)
__device__ KTimer g_ktimer_off;

// ---------------------------------------------------------------------------
// One domain of a batch, in device memory.  The host fills the inputs, the
// options and the output pointers; the block that refines the domain fills
// the results.
// ---------------------------------------------------------------------------
struct Job {
  const double2 *pts;
  const int *tri, *nbr;
  const int2 *seg;
  int np, nt, ns;
  int offcenter, offconstant, mode, pred, placement;
  MlpDev mlp;  // GQM_PLACE_LEARNED: the network on the device
  double theta, max_area;
  long long max_rounds;
  // outputs: each finished domain takes its space from one shared region
  // (bump allocation), so the region holds exactly the batch's results
  char *obase;
  unsigned long long *oused;
  unsigned long long ocap;
  unsigned long long ooff;  // offset of this domain's output block
  // results
  int status, out_np, out_nt, out_ns, rounds;
  long long flip_steps, steiner, midpoints, bad_total, exact_fallbacks, learned_candidates, learned_used;
  double goodcos2;
};

// Capacities of one domain: the logical capacity starts as in the
// single-domain path (refine.cu:6543-6544: pointblock = (int)(0.5 N),
// triblock = 2 pointblock); the physical sizes leave room for four more point
// blocks and five more triangle blocks of growth, and for eight subsegments
// per input segment plus one per two input points.
struct Caps {
  long pointblock, triblock, pphys, tphys, sphys, cav_cap, hsz;
};
__host__ __device__ inline Caps caps_of(int np, int nt, int ns) {
  Caps c;
  c.pointblock = (int)(np * 0.5);
  c.triblock = 2 * c.pointblock;
#ifdef GQM_TEST_TIGHT_BUFFERS
  // test builds: arenas with no room to grow, so that domains overflow and
  // take the single-domain path
  c.pphys = np + c.pointblock;
  c.tphys = nt + c.triblock;
#else
  c.pphys = np + 5 * c.pointblock;
  c.tphys = nt + 6 * c.triblock;
#endif
  c.sphys = 8L * ns + np / 2 + 1024;
  c.cav_cap = c.tphys / 4 + 64;
  c.hsz = 1;
  while (c.hsz < 2L * ns + 16) c.hsz <<= 1;
  return c;
}

// Scratch of one domain, carved from its block's arena.
struct Scratch {
  Mesh M;
  int *emptyt, *bad, *imark, *ilist, *sinks, *wl, *act, *win, *neg, *ll, *sl, *newidx, *tail;
  int *emptyp, *pnew, *enclist, *encl2, *smark, *mids, *snap, *fq, *tl, *cav, *cavn;
  uint8_t *clr;
  double2 *center;
  unsigned long long *hkeys;
  int *hvals, *s2ti;
};
// Walks the arena layout: with base == 0 it only measures (host), otherwise it
// assigns every pointer of S (device).  Every array starts on 256 bytes.
struct Cursor {
  char *base;
  size_t off;
  template <class T>
  __host__ __device__ T *take(long n) {
    off = (off + 255) & ~(size_t)255;
    T *p = reinterpret_cast<T *>(reinterpret_cast<uintptr_t>(base) + off);
    off += sizeof(T) * (size_t)(n > 0 ? n : 1);
    return p;
  }
};
__host__ __device__ inline void carve(Cursor &a, Scratch &S, const Caps &c) {
  const long P = c.pphys, T = c.tphys, Sg = c.sphys;
  Mesh &M = S.M;
  M.pts = a.take<double2>(P);
  M.ps = a.take<uint8_t>(P);
  M.pred = a.take<uint8_t>(P);
  S.emptyp = a.take<int>(P);
  S.pnew = a.take<int>(P);
  S.tail = a.take<int>(P > T ? P : T);
  M.tv = a.take<int4>(T);
  M.tn = a.take<int4>(T);
  M.tsg = a.take<int4>(T);
  M.tst = a.take<uint8_t>(T);
  M.tflip = a.take<uint8_t>(T);
  M.tfo = a.take<uint8_t>(T);
  M.flip0 = a.take<uint8_t>(T);
  S.clr = a.take<uint8_t>(T);
  M.tmark = a.take<int>(T);
  M.tpos = a.take<int>(T);
  M.fstamp = a.take<int>(T);
  M.tstamp = a.take<int>(T);
  M.wbits = a.take<unsigned>(T / 32 + 1);
  M.wcnt = a.take<int>(T / 1024 + 1);
  M.wsup = a.take<int>(T / 32768 + 1);
  M.wmeg = a.take<int>(T / 1048576 + 1);
  S.emptyt = a.take<int>(T);
  S.bad = a.take<int>(T);
  S.imark = a.take<int>(T);
  S.ilist = a.take<int>(T);
  S.sinks = a.take<int>(T);
  S.wl = a.take<int>(T);
  S.act = a.take<int>(T);
  S.win = a.take<int>(T);
  S.neg = a.take<int>(T);
  S.newidx = a.take<int>(T);
  S.fq = a.take<int>(T);
  S.tl = a.take<int>(T);
  S.ll = a.take<int>(2 * T);
  S.sl = a.take<int>(6 * T);
  S.center = a.take<double2>(T);
  M.s2t = a.take<s2t_t>(Sg);
  M.s2seg = a.take<int>(Sg);
  M.enc = a.take<int>(Sg);
  S.enclist = a.take<int>(Sg);
  S.encl2 = a.take<int>(Sg);
  S.smark = a.take<int>(Sg);
  S.mids = a.take<int>(Sg);
  S.snap = a.take<int>(Sg);
  S.cav = a.take<int>((long)kCavityCap * c.cav_cap);
  S.cavn = a.take<int>(c.cav_cap);
  S.hkeys = a.take<unsigned long long>(c.hsz);
  S.hvals = a.take<int>(c.hsz);
  S.s2ti = a.take<int>(c.hsz);
}
// Output block of one finished domain: points, triangles, neighbours,
// segments, point and triangle status bytes, each on 16 bytes.
struct OutLayout {
  unsigned long long pts, tri, nbr, seg, ps, ts, bytes;
};
__host__ __device__ inline unsigned long long up16(unsigned long long x) { return (x + 15) & ~15ull; }
__host__ __device__ inline OutLayout out_layout(long np, long nt, long ns) {
  OutLayout L;
  L.pts = 0;
  L.tri = L.pts + up16(16ull * np);
  L.nbr = L.tri + up16(12ull * nt);
  L.seg = L.nbr + up16(12ull * nt);
  L.ps = L.seg + up16(8ull * ns);
  L.ts = L.ps + up16((unsigned long long)np);
  L.bytes = L.ts + up16((unsigned long long)nt);
  return L;
}
inline size_t arena_bytes(const Caps &c) {
  Cursor a{nullptr, 0};
  Scratch S;
  carve(a, S, c);
  return (a.off + 255) & ~(size_t)255;
}

// ---------------------------------------------------------------------------
// The device-side driver: Refiner (refine.cu) restated for one thread block.
// Every thread runs the same control flow on the same scalars; counts come
// from block-wide compactions or from the shared control block, read after a
// barrier.  Device pointers to counts (the kernels' `dn`) point into shared
// memory.
// ---------------------------------------------------------------------------
enum { C_LIST0 = 0, C_LIST1, C_LIST2, C_MISC };

struct Shared {
  Scratch S;
  FlipCtl fc;
  unsigned long long ctr[6];  // Steiner points, midpoints, -, -, learned candidates, learned points
  double gc[2];
  int cnt[8];
  int scan[33];
  int err;
  int job;
};

template <int PRED>
struct Cta {
  Shared &sh;
  Caps c;
  long pcap, tcap;
  int last_point, last_triangle, last_subseg;
  int nempty_p, nempty_t, lenp, lent;
  int offcenter, offconstant, placement;
  MlpDev mlp;
  long long max_rounds;

  __device__ bool lead() const { return threadIdx.x == 0; }
  template <class F, class Mp>
  __device__ int compact(F f, Mp m, int lo, int hi, int *out) {
    return cta_compact(f, m, lo, hi, out, sh.scan);
  }
  // the device error word, read by every thread before anyone can change it
  // again (the barrier keeps the block's decision on it uniform)
  __device__ int read_err() {
    const int e = sh.err;
    SYNC();
    return e;
  }
  // a count that the next step reads through a pointer
  __device__ int *publish(int slot, int v) {
    if (lead()) sh.cnt[slot] = v;
    SYNC();
    return sh.cnt + slot;
  }

  // updateEmptyPoints / updateEmptyTriangles (refine.cu:149-197)
  __device__ int refresh_points() {
    lenp = compact(PPtDeleted{sh.S.M.ps}, Ident{}, 0, (int)pcap, sh.S.emptyp);
    return lenp;
  }
  __device__ int refresh_tris() {
    lent = compact(PTriNull{sh.S.M.tst}, Ident{}, 0, (int)tcap, sh.S.emptyt);
    return lent;
  }
  // growth steps of refine.cu:3408-3444 / 5259-5296 on the logical capacity
  __device__ int ensure_slots(int npts, int ntris) {
    if (npts > nempty_p) {
      nempty_p = refresh_points();
      long num = 0;
      while (npts > nempty_p + num * c.pointblock) num++;
      if (num) {
        long ncap = pcap + num * c.pointblock;
        if (ncap > c.pphys) return GQM_ERR_ARENA;
        pcap = ncap;
        nempty_p = refresh_points();
      }
    }
    if (ntris > nempty_t) {
      nempty_t = refresh_tris();
      long num = 0;
      while (ntris > nempty_t + num * c.triblock) num++;
      if (num) {
        long ncap = tcap + num * c.triblock;
        if (ncap > c.tphys) return GQM_ERR_ARENA;
        tcap = ncap;
        nempty_t = refresh_tris();
      }
    }
    return GQM_OK;
  }
  // slot bookkeeping after an insertion batch (refine.cu:3545-3559, 5354-5368)
  __device__ void consume_slots(int npts, int ntris) {
    int slot_after = (int)(pcap - last_point);
    int slot_before = nempty_p - slot_after;
    if (slot_before < npts) last_point += npts - slot_before;
    nempty_p -= npts;
    slot_after = (int)(tcap - last_triangle);
    slot_before = nempty_t - slot_after;
    if (slot_before < ntris) last_triangle += ntris - slot_before;
    nempty_t -= ntris;
  }
  __device__ const int *pslots() const { return sh.S.emptyp + (lenp - nempty_p); }
  __device__ const int *tslots() const { return sh.S.emptyt + (lent - nempty_t); }

  // ---- flip-flop (refine.cu:2328-2490): the steps of refine.cu's flip graph ----
  __device__ int flip_flop(int ntri) {
    Scratch &S = sh.S;
    FlipCtl *fc = &sh.fc;
    k_flip_entry_reset(S.M, ntri);
    SYNC();
    int n = compact(PNotNullFlag{S.M.tst, S.M.tflip}, Ident{}, 0, ntri, S.act);
    if (lead()) {
      fc->nact = n;
      fc->nact_next = 0;
      fc->entry_steps = fc->steps;
      flip_next(fc);
    }
    SYNC();
    while (fc->cond) {
      FlipQ Q{S.fq, &fc->qn, &fc->gen};
      TouchL T{S.tl, &fc->tn, &fc->gen};
      k_check_flip2<PRED>(S.M, S.act, &fc->nact, S.clr, T, &g_ktimer_off);
      SYNC();
      k_flip_winner2(S.M, S.act, &fc->nact, S.clr, Q, S.win, &fc->winn);
      SYNC();
      k_link_phase1(S.M, S.win, &fc->winn, S.ll, S.sl, &fc->epoch);
      SYNC();
      k_phase2(S.M, S.win, &fc->winn, S.ll, S.sl);
      SYNC();
      k_phase3q(S.M, S.win, &fc->winn, S.sl, Q);
      SYNC();
      k_mark_red_steiner_q(S.M, S.tl, &fc->tn, Q);
      SYNC();
      k_flip_reset_filter(S.M, S.tl, &fc->tn, S.fq, &fc->qn, S.act, &fc->nact_next);
      SYNC();
      if (lead()) {
        fc->nact = fc->nact_next;
        fc->nact_next = 0;
        flip_next(fc);
      }
      SYNC();
    }
    return GQM_OK;  // errors raised on the device are read by the round loop
  }

  // ---- splitEncsegs (refine.cu:3180-3778) ----
  __device__ int split_encsegs() {
    Scratch &S = sh.S;
    long long outer = 0;
    for (;;) {
      int nenc = compact(PNonNeg{S.M.enc}, Ident{}, 0, last_subseg, S.enclist);
      if (nenc == 0) break;
      if (++outer > max_rounds) return GQM_ERR_ROUND_LIMIT;
      // delete free Steiner points inside diametral circles
      cta_copy(S.smark, S.enclist, nenc);
      SYNC();
      int nmark = nenc;
      long long inner = 0;
      for (;;) {
        int ndel = compact(PNonNeg{S.smark}, ValueOf{S.smark}, 0, nmark, S.mids);
        if (ndel == 0) break;
        if (++inner > max_rounds) return GQM_ERR_ROUND_LIMIT;
        nmark = ndel;
        k_mark_redundant(S.M, S.smark, S.mids, publish(C_LIST1, ndel));
        SYNC();
        int rc = flip_flop(last_triangle);
        if (rc) return rc;
      }
      int rc = ensure_slots(nenc, 2 * nenc);
      if (rc) return rc;
      if (last_subseg + nenc > c.sphys) return GQM_ERR_ARENA;
      cta_fill(S.M.enc + last_subseg, nenc, -1);
      cta_copy(S.smark, S.enclist, nenc);
      SYNC();
      long long mid_iter = 0;
      for (;;) {
        int nmid = compact(PNonNeg{S.smark}, Ident{}, 0, nenc, S.mids);
        if (nmid == 0) break;
        if (++mid_iter > 64 * max_rounds) return GQM_ERR_ROUND_LIMIT;
        int *dn = publish(C_LIST1, nmid);
        k_reset_mid(S.M, S.mids, dn, S.smark);
        SYNC();
        k_mark_mid(S.M, S.mids, dn, S.smark);
        SYNC();
        k_mid_snapshot(S.M, S.mids, dn, S.smark, S.snap);
        if (lead()) sh.fc.epoch++;
        SYNC();
        k_insert_mid(S.M, S.mids, dn, S.smark, S.snap, pslots(), tslots(), last_subseg, &sh.fc.epoch, sh.ctr + 1);
        SYNC();
        k_update_mid_nbrs(S.M, S.mids, dn, S.smark, S.enclist);
        SYNC();
      }
      consume_slots(nenc, 2 * nenc);
      last_subseg += nenc;
      rc = flip_flop(last_triangle);
      if (rc) return rc;
    }
    return GQM_OK;
  }

  // ---- splitTriangles (refine.cu:5107-5547) ----
  __device__ int split_triangles(int nbad) {
    Scratch &S = sh.S;
    int *dn = sh.cnt + C_LIST2;  // number of bad triangles, published by the caller
    cta_copy(S.imark, S.bad, nbad);
    cta_copy(S.ilist, S.bad, nbad);
    k_circumcenter(S.M, S.bad, dn, (double)offconstant, offcenter, S.center);
    cta_fill(S.M.tmark, last_triangle, kMaxInt);
    SYNC();
    if (placement == GQM_PLACE_LEARNED) {
      k_learned_place(S.M, S.bad, dn, mlp, S.center, sh.ctr + 4);
      SYNC();
    }
    k_locate<PRED>(S.M, S.bad, dn, S.center, S.sinks);
    SYNC();
    k_remove_losers(S.M, S.bad, dn, S.sinks, S.imark);
    SYNC();
    cta_fill(S.M.tmark, last_triangle, kMaxInt);
    SYNC();
    if (nbad > c.cav_cap) return GQM_ERR_ARENA;
    k_cavity_mark<PRED>(S.M, dn, S.sinks, S.center, S.imark, S.ilist, S.cav, S.cavn, nbad);
    SYNC();
    k_cavity_check(S.M, dn, S.cav, S.cavn, nbad, S.imark, S.ilist);
    SYNC();
    int nst = compact(PNonNeg{S.imark}, Ident{}, 0, nbad, S.wl);
    int *dw = publish(C_LIST1, nst);
    cta_fill(S.encl2, last_subseg, -1);
    SYNC();
    k_mark_onsegs(S.M, S.wl, dw, S.sinks, S.encl2);
    SYNC();
    int rc = ensure_slots(nst, 2 * nst);
    if (rc) return rc;
    k_reset_steiner(S.M, S.wl, dw, S.sinks);
    if (lead()) sh.fc.epoch++;
    SYNC();
    k_insert_steiner(S.M, S.wl, dw, S.sinks, S.center, pslots(), tslots(), &sh.fc.epoch, sh.ctr + 0);
    SYNC();
    k_update_steiner_nbrs(S.M, S.wl, dw, S.sinks);
    SYNC();
    consume_slots(nst, 2 * nst);
    rc = flip_flop(last_triangle);
    if (rc) return rc;
    k_onsegs_to_enc(S.M, S.encl2, last_subseg);
    SYNC();
    return GQM_OK;
  }

  // ---- output compaction (refine.cu:5758-6428) ----
  __device__ void compact_output(int &out_np, int &out_nt) {
    Scratch &S = sh.S;
    int newn = compact(PTriLive{S.M.tst}, Ident{}, 0, last_triangle, S.tail);
    k_newidx_init(S.M, S.newidx, last_triangle, newn, S.M.tst, (uint8_t)TS_NOTNULL, false);
    SYNC();
    if (newn < last_triangle) {
      compact(PTriNull{S.M.tst}, Ident{}, 0, newn, S.emptyt);
      int nmove = compact(PTriLive{S.M.tst}, Ident{}, newn, last_triangle, S.tail);
      k_compact_tris_move(S.M, S.tail, S.emptyt, publish(C_LIST1, nmove), S.newidx);
      SYNC();
      k_fix_nbrs(S.M, S.newidx, newn);
      k_fix_s2t(S.M, S.newidx, last_subseg);
      SYNC();
    }
    int ntri = newn;
    int newp = compact(PPtLive{S.M.ps}, Ident{}, 0, last_point, S.pnew);
    k_newidx_init(S.M, S.pnew, last_point, newp, S.M.ps, (uint8_t)PS_DELETED, true);
    SYNC();
    if (newp < last_point) {
      compact(PPtDeleted{S.M.ps}, Ident{}, 0, newp, S.emptyp);
      int nmove = compact(PPtLive{S.M.ps}, Ident{}, newp, last_point, S.tail);
      k_compact_pts_move(S.M, S.tail, S.emptyp, publish(C_LIST1, nmove), S.pnew);
      SYNC();
      k_fix_tri_vertices(S.M, S.pnew, ntri);
      SYNC();
    }
    out_np = newp;
    out_nt = ntri;
  }

  // ---- the whole refinement of one domain (Refiner::run) ----
  __device__ int run(Job &J) {
    Scratch &S = sh.S;
    const int np = J.np, nt = J.nt, ns = J.ns;
    c = caps_of(np, nt, ns);
    offcenter = J.offcenter;
    offconstant = J.offconstant;
    placement = J.placement;
    mlp = J.mlp;
    max_rounds = J.max_rounds;
    pcap = np + c.pointblock;
    tcap = nt + c.triblock;
    if (lead()) {
      S.M.segs = J.seg;
      S.M.err = &sh.err;
      sh.err = 0;
      for (int i = 0; i < 6; ++i) sh.ctr[i] = 0;
      FlipCtl &fc = sh.fc;
      fc.gen = 0;
      fc.epoch = 0;
      fc.steps = 0;
      fc.entry_steps = 0;
      fc.cap_hit = 0;
      fc.cond = 0;
      fc.cap = 64 * max_rounds;
      fc.errp = &sh.err;
      for (int b = 0; b < kFlipProfileBins; ++b) fc.prof_steps[b] = fc.prof_items[b] = 0;
    }
    SYNC();
    // stamps, tags and winner counts start from zero for every domain
    cta_fill(S.M.s2t, c.sphys, (s2t_t)0);
    cta_fill(S.M.fstamp, c.tphys, 0);
    cta_fill(S.M.tstamp, c.tphys, 0);
    cta_fill(S.M.wbits, c.tphys / 32 + 1, 0u);
    cta_fill(S.M.wcnt, c.tphys / 1024 + 1, 0);
    cta_fill(S.M.wsup, c.tphys / 32768 + 1, 0);
    cta_fill(S.M.wmeg, c.tphys / 1048576 + 1, 0);
    k_check_input(J.pts, np, J.tri, J.nbr, nt, reinterpret_cast<const int *>(J.seg), ns, &sh.err);
    k_goodcos(J.theta, sh.gc);
    SYNC();
    if (const int e = read_err()) return e;
    if (lead()) {
      S.M.gc2 = sh.gc[0];
      S.M.mode = J.mode;
      S.M.max_area = J.max_area;
      J.goodcos2 = sh.gc[0];
    }
    SYNC();
    k_init_points(S.M, J.pts, np, (int)c.pphys);
    k_init_tris(S.M, J.tri, J.nbr, nt, (int)c.tphys);
    cta_fill(S.hkeys, c.hsz, ~0ull);
    cta_fill(S.s2ti, (long)ns + 1, -1);
    SYNC();
    // initSubsegs via a hash of segment endpoints
    k_seg_hash_insert(J.seg, ns, S.hkeys, S.hvals, (unsigned)(c.hsz - 1));
    SYNC();
    k_init_subsegs(S.M, nt, S.hkeys, S.hvals, (unsigned)(c.hsz - 1), S.s2ti);
    SYNC();
    k_pack_s2t(S.M, S.s2ti, ns);
    SYNC();
    last_point = np;
    last_triangle = nt;
    last_subseg = ns;
    nempty_p = refresh_points();
    nempty_t = refresh_tris();
    k_mark_all_encsegs(S.M, ns);
    SYNC();
    int rc = split_encsegs();
    int rounds = 0;
    long long bad_total = 0;
    while (rc == 0) {
      k_mark_bad(S.M, last_triangle);
      SYNC();
      int nbad = compact(PBad{S.M.tst}, Ident{}, 0, last_triangle, S.bad);
      publish(C_LIST2, nbad);
      if (const int e = read_err()) {
        rc = e;
        break;
      }
      if (nbad == 0) break;
      if (rounds >= max_rounds) {
        rc = GQM_ERR_ROUND_LIMIT;
        break;
      }
      bad_total += nbad;
      rc = split_triangles(nbad);
      if (rc) break;
      rc = split_encsegs();
      if (rc) break;
      k_points_old(S.M, last_point);
      SYNC();
      rounds++;
    }
    if (const int e = read_err()) rc = rc ? rc : e;
    int out_np = 0, out_nt = 0;
    if (rc == 0) compact_output(out_np, out_nt);
    if (const int e = read_err()) rc = rc ? rc : e;
    if (rc == 0) {
      const OutLayout L = out_layout(out_np, out_nt, last_subseg);
      if (lead()) {
        const unsigned long long off = atomicAdd(J.oused, (unsigned long long)L.bytes);
        sh.cnt[C_MISC] = off + L.bytes <= J.ocap ? 0 : GQM_ERR_ARENA;
        J.ooff = off;
      }
      SYNC();
      rc = sh.cnt[C_MISC];
      if (rc == 0) {
        char *o = J.obase + J.ooff;
        k_emit_output(S.M, out_nt, last_subseg, reinterpret_cast<int *>(o + L.tri), reinterpret_cast<int *>(o + L.nbr),
                      reinterpret_cast<int *>(o + L.seg), reinterpret_cast<uint8_t *>(o + L.ts));
        k_emit_pstatus(S.M, out_np, reinterpret_cast<uint8_t *>(o + L.ps));
        double2 *op = reinterpret_cast<double2 *>(o + L.pts);
        for (int i = (int)threadIdx.x; i < out_np; i += (int)blockDim.x) op[i] = S.M.pts[i];
      }
      SYNC();
    }
    if (lead()) {
      J.out_np = out_np;
      J.out_nt = out_nt;
      J.out_ns = last_subseg;
      J.rounds = rounds;
      J.bad_total = bad_total;
      J.flip_steps = sh.fc.steps;
      J.steiner = (long long)sh.ctr[0];
      J.midpoints = (long long)sh.ctr[1];
      J.exact_fallbacks = (long long)sh.ctr[2];
      J.learned_candidates = (long long)sh.ctr[4];
      J.learned_used = (long long)sh.ctr[5];
    }
    return rc;
  }
};

// The persistent batch kernel: each block takes the next domain (largest
// first) until the queue is empty, refining it in its own arena.
template <int PRED>
__device__ void batch_body(Job *jobs, const int *order, int njobs, int *next, char *arenas, size_t arena_stride,
                           Shared &sh) {
  char *arena = arenas + (size_t)blockIdx.x * arena_stride;
  for (;;) {
    if (threadIdx.x == 0) sh.job = atomicAdd(next, 1);
    SYNC();
    const int k = sh.job;
    SYNC();
    if (k >= njobs) break;
    Job &J = jobs[order[k]];
    if (threadIdx.x == 0) {
      Cursor a{arena, 0};
      carve(a, sh.S, caps_of(J.np, J.nt, J.ns));
    }
    SYNC();
    Cta<PRED> R{sh};
    const int rc = R.run(J);
    SYNC();
    if (threadIdx.x == 0) J.status = rc;
  }
}
template <int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_batch(Job *jobs, const int *order, int njobs, int *next, char *arenas,
                                                    size_t arena_stride, int pred) {
  __shared__ Shared sh;
  if (pred)
    batch_body<1>(jobs, order, njobs, next, arenas, arena_stride, sh);
  else
    batch_body<0>(jobs, order, njobs, next, arenas, arena_stride, sh);
}

// ---------------------------------------------------------------------------
// Small flip steps of the single-domain engine
// ---------------------------------------------------------------------------
// The single-domain flip-flop loop (refine.cu's flip graph: one launch per
// step phase) spends most of its steps on small active sets: on the 2M-point
// input three quarters of the steps have fewer than 2,048 triangles, where the
// eight launches of a step cost more than the work.  This kernel runs in the
// loop body after the step's condition kernel: while the next step's active
// set has at most `limit` triangles, one block runs whole steps (the same
// phases, compiled in block mode, separated by barriers), then it re-sets the
// loop condition.  The steps and their results are the ones the grid kernels
// would produce (every phase is decided by the reference's rules, not by the
// thread layout).  The loop's control block (list lengths, stamps'
// generation, launch epoch) is worked on in shared memory and written back
// at exit: a step of a few triangles is a chain of dependent memory accesses,
// and every counter read or atomic on shared memory instead of global memory
// takes one L2 round trip out of that chain.
constexpr int kSmallThreads = 512;
template <int PRED>
__global__ void __launch_bounds__(kSmallThreads, 1)
    k_flip_small(Mesh M, FlipCtl *gfc, int *act, uint8_t *clr, int *win, int *ll, int *sl, int *fq, int *tl,
                 int limit, cudaGraphConditionalHandle h, int graph, KTimer *tm) {
  __shared__ int go;
  __shared__ FlipCtl sfc;
  FlipCtl *fc = &sfc;
  if (threadIdx.x == 0) sfc = *gfc;
  const int timed = tm->on;
  const unsigned long long start = timed ? global_ns() : 0;
  long long items = 0, wins = 0;  // thread 0's count of the launch's work (probe only)
  for (;;) {
    if (threadIdx.x == 0) go = fc->cond && fc->nact <= limit;
    SYNC();
    if (!go) break;
    if (threadIdx.x == 0) items += fc->nact;
    FlipQ Q{fq, &fc->qn, &fc->gen};
    TouchL T{tl, &fc->tn, &fc->gen};
    k_check_flip2<PRED>(M, act, &fc->nact, clr, T, &g_ktimer_off);
    SYNC();
    k_flip_winner2(M, act, &fc->nact, clr, Q, win, &fc->winn);
    SYNC();
    if (threadIdx.x == 0) wins += fc->winn;
    k_link_phase1(M, win, &fc->winn, ll, sl, &fc->epoch);
    SYNC();
    k_phase2(M, win, &fc->winn, ll, sl);
    SYNC();
    k_phase3q(M, win, &fc->winn, sl, Q);
    SYNC();
    k_mark_red_steiner_q(M, tl, &fc->tn, Q);
    SYNC();
    k_flip_reset_filter(M, tl, &fc->tn, fq, &fc->qn, act, &fc->nact_next);
    SYNC();
    if (threadIdx.x == 0) {
      fc->nact = fc->nact_next;
      fc->nact_next = 0;
      fc->small_steps++;
      flip_next(fc);
    }
    SYNC();
  }
  if (threadIdx.x == 0) *gfc = sfc;
#ifndef GQM_HOST_EMU
  if (graph && threadIdx.x == 0) cudaGraphSetConditional(h, fc->cond);
#endif
  (void)h;
  (void)graph;
  if (timed) ktimer_end(tm, start, items, wins);
}

}  // namespace gqm

// Launch of k_flip_small on the single-domain engine's buffers (refine.cu).
// mesh points at the caller's Mesh (the same layout in both compilations);
// timer is the caller's KTimer (the same layout too).
int gqm_flip_small_launch(const void *mesh, size_t mesh_bytes, void *fc, int pred, int *act, uint8_t *clr, int *win,
                          int *ll, int *sl, int *fq, int *tl, int limit, cudaStream_t st,
                          cudaGraphConditionalHandle h, int graph, void *timer) {
  if (mesh_bytes != sizeof(gqm::Mesh)) return GQM_ERR_ARGUMENT;
  gqm::Mesh M;
  memcpy(&M, mesh, sizeof(M));
  gqm::FlipCtl *c = static_cast<gqm::FlipCtl *>(fc);
  gqm::KTimer *tm = static_cast<gqm::KTimer *>(timer);
#ifdef GQM_HOST_EMU
  (void)st;
  if (pred)
    gqm::k_flip_small<1>(M, c, act, clr, win, ll, sl, fq, tl, limit, h, graph, tm);
  else
    gqm::k_flip_small<0>(M, c, act, clr, win, ll, sl, fq, tl, limit, h, graph, tm);
#else
  if (pred)
    gqm::k_flip_small<1><<<1, gqm::kSmallThreads, 0, st>>>(M, c, act, clr, win, ll, sl, fq, tl, limit, h, graph, tm);
  else
    gqm::k_flip_small<0><<<1, gqm::kSmallThreads, 0, st>>>(M, c, act, clr, win, ll, sl, fq, tl, limit, h, graph, tm);
#endif
  return GQM_OK;
}

// The incircle expansion-fallback counter of this translation unit's kernels
// (a device variable exists once per translation unit): added to *sum, then
// zeroed when `reset` is set.  Called by the single-domain driver, which
// reports the counters of all its kernels together.
int gqm_fallbacks_cta(unsigned long long *sum, int reset, cudaStream_t st) {
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

// ===========================================================================
// Host side
// ===========================================================================
namespace gqm {
namespace {

typedef void (*BatchFn)(Job *, const int *, int, int *, char *, size_t, int);
struct Variant {
  int threads, minb;
  BatchFn fn;
};
// compiled (threads per block, blocks per SM) pairs; the autotuner picks one
const Variant kVariants[] = {{128, 4, k_batch<128, 4>}, {256, 1, k_batch<256, 1>}, {256, 2, k_batch<256, 2>},
                             {512, 1, k_batch<512, 1>}};
constexpr int kNumVariants = (int)(sizeof(kVariants) / sizeof(kVariants[0]));
constexpr int kDefaultVariant = 2;

// Buffers kept per device between calls (grow only).
struct DevCache {
  std::mutex mu;
  bool init = false;
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  char *d_in = nullptr, *d_out = nullptr, *d_arena = nullptr, *h_in = nullptr, *h_out = nullptr;
  size_t in_cap = 0, out_cap = 0, arena_cap = 0, h_in_cap = 0, h_out_cap = 0;
  Job *d_jobs = nullptr;
  int *d_order = nullptr;
  int jobs_cap = 0;
  int *d_next = nullptr;
  unsigned long long *d_used = nullptr;
  int tuned = -1;  // autotuned variant, -1 until gqm_batch_autotune ran
  int sms = 148;
};
DevCache g_dev[16];

template <class T>
int grow_dev(T **p, size_t *cap, size_t need) {
  if (need <= *cap) return GQM_OK;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  if (cudaMalloc((void **)p, need) != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    return GQM_ERR_MEMORY;
  }
  *cap = need;
  return GQM_OK;
}
int grow_host(char **p, size_t *cap, size_t need) {
  if (need <= *cap) return GQM_OK;
  if (*p) cudaFreeHost(*p);
  *p = nullptr;
  *cap = 0;
  if (cudaMallocHost((void **)p, need) != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    return GQM_ERR_MEMORY;
  }
  *cap = need;
  return GQM_OK;
}
size_t up256(size_t x) { return (x + 255) & ~(size_t)255; }

// f(k) for k in [0, n) on the host's cores (packing and unpacking of the
// domains' arrays are independent memcpy's)
template <class F>
void parallel_for(int n, F f) {
  int nt = (int)std::thread::hardware_concurrency();
  nt = std::max(1, std::min(nt, 32));
  if (n < 64 || nt == 1) {
    for (int k = 0; k < n; ++k) f(k);
    return;
  }
  std::vector<std::thread> pool;
  for (int t = 0; t < nt; ++t)
    pool.emplace_back([&, t] {
      for (int k = t; k < n; k += nt) f(k);
    });
  for (auto &th : pool) th.join();
}

int check_domain(const gqm_cdt_in *in, const gqm_options *opt) {
  if (!in || !opt) return GQM_ERR_ARGUMENT;
  if (in->numberofpoints < 3 || in->numberoftriangles < 1 || in->numberofsegments < 0) return GQM_ERR_ARGUMENT;
  if (!in->pointlist || !in->trianglelist || !in->neighborlist) return GQM_ERR_ARGUMENT;
  if (in->numberofsegments > 0 && !in->segmentlist) return GQM_ERR_ARGUMENT;
  if (!(opt->theta > 0.0 && opt->theta < 60.0)) return GQM_ERR_ARGUMENT;
  if (opt->placement != GQM_PLACE_PLAIN && (opt->placement != GQM_PLACE_LEARNED || !opt->mlp)) return GQM_ERR_ARGUMENT;
  if (!(opt->max_area >= 0.0)) return GQM_ERR_ARGUMENT;
  return GQM_OK;
}

double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// One persistent batch over the domains `ids` (all with the same predicate
// mode) with kernel variant `var`.  Results of domains that finished land in
// out/stats; the status of each domain in status[d].
int run_batch(DevCache &C, const std::vector<int> &ids, const gqm_cdt_in *in, gqm_cdt_out *out,
              const gqm_options *opt, gqm_stats *stats, int var, double mem_fraction, int *status,
              gqm_batch_report *rep, bool keep_outputs) {
  const int n = (int)ids.size();
  if (n == 0) return GQM_OK;
  auto t0 = std::chrono::steady_clock::now();
  // sizes
  std::vector<size_t> in_off(n);
  size_t in_bytes = 0, arena = 0;
  unsigned long long out_bound = 0;
  for (int k = 0; k < n; ++k) {
    const gqm_cdt_in &d = in[ids[k]];
    in_off[k] = in_bytes;
    in_bytes += up256(16ull * d.numberofpoints) + 2 * up256(12ull * d.numberoftriangles) +
                up256(8ull * d.numberofsegments);
    const Caps c = caps_of(d.numberofpoints, d.numberoftriangles, d.numberofsegments);
    arena = std::max(arena, arena_bytes(c));
    out_bound += out_layout(c.pphys, c.tphys, c.sphys).bytes;
  }
  // grid: resident blocks of the variant, bounded by the domains and memory
  const Variant &V = kVariants[var];
  int per_sm = V.minb;
#ifndef GQM_HOST_EMU
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, V.fn, V.threads, 0) == cudaSuccess && occ > 0)
    per_sm = occ;
  else
    cudaGetLastError();
#endif
  long grid = std::min<long>((long)C.sms * per_sm, n);
#ifndef GQM_HOST_EMU
  size_t freeb = 0, totb = 0;
  cudaMemGetInfo(&freeb, &totb);
  const size_t have = (size_t)(mem_fraction * (double)(freeb + C.in_cap + C.out_cap + C.arena_cap));
  const size_t fixed = up256(in_bytes) + up256(out_bound);
  if (fixed + arena > have) return GQM_ERR_MEMORY;
  grid = std::min<long>(grid, (long)((have - fixed) / arena));
#else
  (void)mem_fraction;
  grid = 1;
#endif
  if (grid < 1) return GQM_ERR_MEMORY;
  if (grow_dev(&C.d_in, &C.in_cap, in_bytes) || grow_dev(&C.d_out, &C.out_cap, out_bound) ||
      grow_dev(&C.d_arena, &C.arena_cap, arena * (size_t)grid) || grow_host(&C.h_in, &C.h_in_cap, in_bytes))
    return GQM_ERR_MEMORY;
  if (n > C.jobs_cap) {
    if (C.d_jobs) cudaFree(C.d_jobs);
    if (C.d_order) cudaFree(C.d_order);
    C.d_jobs = nullptr;
    C.d_order = nullptr;
    C.jobs_cap = 0;
    if (cudaMalloc((void **)&C.d_jobs, sizeof(Job) * n) != cudaSuccess ||
        cudaMalloc((void **)&C.d_order, sizeof(int) * n) != cudaSuccess)
      return GQM_ERR_MEMORY;
    C.jobs_cap = n;
  }
  // inputs packed into pinned memory on the host's cores and uploaded in
  // pieces of 32 MB, the front while the back is packed
  std::vector<Job> jobs(n);
  {
    std::vector<HostCopy> parts;
    parts.reserve(4 * (size_t)n);
    for (int k = 0; k < n; ++k) {
      const gqm_cdt_in &D = in[ids[k]];
      char *h = C.h_in + in_off[k];
      const size_t bp = up256(16ull * D.numberofpoints), bt = up256(12ull * D.numberoftriangles);
      parts.push_back({h, D.pointlist, 16ull * D.numberofpoints});
      parts.push_back({h + bp, D.trianglelist, 12ull * D.numberoftriangles});
      parts.push_back({h + bp + bt, D.neighborlist, 12ull * D.numberoftriangles});
      if (D.numberofsegments) parts.push_back({h + bp + 2 * bt, D.segmentlist, 8ull * D.numberofsegments});
    }
    host_copy_streamed(parts, C.h_in, 32u << 20, [&](size_t off, size_t bytes) {
      cudaMemcpyAsync(C.d_in + off, C.h_in + off, bytes, cudaMemcpyHostToDevice, C.st);
    });
  }
  for (int k = 0; k < n; ++k) {
    const int d = ids[k];
    const gqm_cdt_in &D = in[d];
    char *g = C.d_in + in_off[k];
    const size_t bp = up256(16ull * D.numberofpoints), bt = up256(12ull * D.numberoftriangles);
    Job &J = jobs[k];
    memset(&J, 0, sizeof(J));
    J.pts = reinterpret_cast<const double2 *>(g);
    J.tri = reinterpret_cast<const int *>(g + bp);
    J.nbr = reinterpret_cast<const int *>(g + bp + bt);
    J.seg = reinterpret_cast<const int2 *>(g + bp + 2 * bt);
    J.np = D.numberofpoints;
    J.nt = D.numberoftriangles;
    J.ns = D.numberofsegments;
    const gqm_options &o = opt[d];
    J.theta = o.theta;
    J.max_area = o.max_area > 0.0 ? o.max_area : 0.0;
    J.mode = o.mode ? 1 : 0;
    J.pred = o.predicates ? 1 : 0;
    J.max_rounds = o.max_rounds > 0 ? o.max_rounds : 1000000;
    J.offcenter = 0;
    double offc = 0.0;
    if (o.insert_policy == GQM_OFFCENTER) {  // refine.cu:6555-6567, evaluated on the host as there
      J.offcenter = 1;
      const double cg = cos(o.theta * GQM_PI / 180);
      offc = 0.475 * sqrt((1.0 + cg) / (1.0 - cg));
    }
    J.offconstant = (int)offc;
    J.obase = C.d_out;
    J.oused = C.d_used;
    J.ocap = out_bound;
    J.status = GQM_ERR_CUDA;  // overwritten by the block that refines it
  }
  // networks of the learned placement: one device copy per distinct array
  std::vector<const float *> nets;
  for (int k = 0; k < n; ++k) {
    const gqm_options &o = opt[ids[k]];
    if (o.placement == GQM_PLACE_LEARNED && std::find(nets.begin(), nets.end(), o.mlp) == nets.end())
      nets.push_back(o.mlp);
  }
  char *dnet = nullptr;
  const size_t net_bytes = up256(sizeof(uint16_t) * kMlpW) + up256(sizeof(float) * kMlpB);
  if (!nets.empty()) {
    if (cudaMalloc((void **)&dnet, net_bytes * nets.size()) != cudaSuccess) return GQM_ERR_MEMORY;
    std::vector<char> h(net_bytes * nets.size());
    for (size_t i = 0; i < nets.size(); ++i)
      mlp_pack(nets[i], reinterpret_cast<uint16_t *>(h.data() + i * net_bytes),
               reinterpret_cast<float *>(h.data() + i * net_bytes + up256(sizeof(uint16_t) * kMlpW)));
    cudaMemcpy(dnet, h.data(), h.size(), cudaMemcpyHostToDevice);
  }
  for (int k = 0; k < n; ++k) {
    const gqm_options &o = opt[ids[k]];
    jobs[k].placement = o.placement == GQM_PLACE_LEARNED ? GQM_PLACE_LEARNED : GQM_PLACE_PLAIN;
    if (jobs[k].placement == GQM_PLACE_LEARNED) {
      const size_t i = (size_t)(std::find(nets.begin(), nets.end(), o.mlp) - nets.begin());
      char *base = dnet + i * net_bytes;
      jobs[k].mlp = mlp_dev(reinterpret_cast<uint16_t *>(base),
                            reinterpret_cast<float *>(base + up256(sizeof(uint16_t) * kMlpW)));
    }
  }
  // largest first
  std::vector<int> order(n);
  for (int k = 0; k < n; ++k) order[k] = k;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return jobs[a].np > jobs[b].np; });
  cudaMemcpyAsync(C.d_jobs, jobs.data(), sizeof(Job) * n, cudaMemcpyHostToDevice, C.st);
  cudaMemcpyAsync(C.d_order, order.data(), sizeof(int) * n, cudaMemcpyHostToDevice, C.st);
  cudaMemsetAsync(C.d_next, 0, sizeof(int), C.st);
  cudaMemsetAsync(C.d_used, 0, sizeof(unsigned long long), C.st);
  if (cudaStreamSynchronize(C.st) != cudaSuccess) return GQM_ERR_CUDA;
  const double h2d = ms_since(t0);
  // the persistent launch
  cudaEventRecord(C.e0, C.st);
#ifdef GQM_HOST_EMU
  V.fn(C.d_jobs, C.d_order, n, C.d_next, C.d_arena, arena, jobs[0].pred);
#else
  V.fn<<<(unsigned)grid, V.threads, 0, C.st>>>(C.d_jobs, C.d_order, n, C.d_next, C.d_arena, arena, jobs[0].pred);
#endif
  cudaEventRecord(C.e1, C.st);
  if (cudaStreamSynchronize(C.st) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
    if (dnet) cudaFree(dnet);
    return GQM_ERR_CUDA;
  }
  float kms = 0.0f;
  cudaEventElapsedTime(&kms, C.e0, C.e1);
  if (dnet) cudaFree(dnet);
  // results: the job table, then the used part of the output region
  auto t1 = std::chrono::steady_clock::now();
  unsigned long long used = 0;
  cudaMemcpy(jobs.data(), C.d_jobs, sizeof(Job) * n, cudaMemcpyDeviceToHost);
  cudaMemcpy(&used, C.d_used, sizeof(used), cudaMemcpyDeviceToHost);
  // a large output region is downloaded straight into a pinned block that the
  // domains' results share (released by the last gqm_free_result); a smaller
  // one through the staging buffer into malloc()ed arrays
  char *blk = nullptr;
  if (keep_outputs) {
    int nres = 0;
    for (int k = 0; k < n; ++k) nres += jobs[k].status == GQM_OK;
    blk = gqm_pinned_take((size_t)used, nres);
    if (blk) {
      if (cudaMemcpy(blk, C.d_out, (size_t)used, cudaMemcpyDeviceToHost) != cudaSuccess) {
        for (int k = 0; k < nres; ++k) gqm_pinned_give(blk);
        return GQM_ERR_CUDA;
      }
    } else {
      if (grow_host(&C.h_out, &C.h_out_cap, (size_t)used)) return GQM_ERR_MEMORY;
      if (used && cudaMemcpy(C.h_out, C.d_out, (size_t)used, cudaMemcpyDeviceToHost) != cudaSuccess)
        return GQM_ERR_CUDA;
    }
  }
  int alloc_fail = 0;
  for (int k = 0; k < n; ++k) {
    const int d = ids[k];
    const Job &J = jobs[k];
    status[d] = J.status;
    if (J.status != GQM_OK) continue;
    if (stats) {
      gqm_stats &s = stats[d];
      memset(&s, 0, sizeof(s));
      s.rounds = J.rounds;
      s.flip_steps = J.flip_steps;
      s.steiner_inserted = J.steiner;
      s.midpoints_inserted = J.midpoints;
      s.bad_total = J.bad_total;
      s.exact_fallbacks = J.exact_fallbacks;
      s.learned_candidates = J.learned_candidates;
      s.learned_used = J.learned_used;
      s.goodcos2 = J.goodcos2;
      s.kernel_launches = 1;
      s.device_ms = kms;
    }
    if (!keep_outputs) continue;
    gqm_cdt_out &R = out[d];
    R.numberofpoints = J.out_np;
    R.numberoftriangles = J.out_nt;
    R.numberofsegments = J.out_ns;
    if (blk) {
      const OutLayout L = out_layout(J.out_np, J.out_nt, J.out_ns);
      char *o = blk + J.ooff;
      R.pointlist = reinterpret_cast<double *>(o + L.pts);
      R.trianglelist = reinterpret_cast<int *>(o + L.tri);
      R.neighborlist = reinterpret_cast<int *>(o + L.nbr);
      R.segmentlist = reinterpret_cast<int *>(o + L.seg);
      R.pstatus = reinterpret_cast<unsigned char *>(o + L.ps);
      R.tstatus = reinterpret_cast<unsigned char *>(o + L.ts);
      continue;
    }
    R.pointlist = (double *)malloc(16ull * J.out_np + 16);
    R.trianglelist = (int *)malloc(12ull * J.out_nt + 16);
    R.neighborlist = (int *)malloc(12ull * J.out_nt + 16);
    R.segmentlist = (int *)malloc(8ull * J.out_ns + 16);
    R.pstatus = (unsigned char *)malloc((size_t)J.out_np + 16);
    R.tstatus = (unsigned char *)malloc((size_t)J.out_nt + 16);
    if (!R.pointlist || !R.trianglelist || !R.neighborlist || !R.segmentlist || !R.pstatus || !R.tstatus)
      alloc_fail = 1;
  }
  if (alloc_fail) return GQM_ERR_MEMORY;  // the caller releases every out[]
  if (keep_outputs && !blk)
    parallel_for(n, [&](int k) {
      const Job &J = jobs[k];
      if (J.status != GQM_OK) return;
      const OutLayout L = out_layout(J.out_np, J.out_nt, J.out_ns);
      const char *o = C.h_out + J.ooff;
      gqm_cdt_out &R = out[ids[k]];
      memcpy(R.pointlist, o + L.pts, 16ull * J.out_np);
      memcpy(R.trianglelist, o + L.tri, 12ull * J.out_nt);
      memcpy(R.neighborlist, o + L.nbr, 12ull * J.out_nt);
      memcpy(R.segmentlist, o + L.seg, 8ull * J.out_ns);
      memcpy(R.pstatus, o + L.ps, (size_t)J.out_np);
      memcpy(R.tstatus, o + L.ts, (size_t)J.out_nt);
    });
  if (rep) {
    rep->grid = (int)grid;
    rep->threads_per_block = V.threads;
    rep->blocks_per_sm = V.minb;
    rep->arena_bytes = (long long)arena;
    rep->kernel_ms += kms;
    rep->h2d_ms += h2d;
    rep->d2h_ms += ms_since(t1);
  }
  return GQM_OK;
}

int setup_dev(DevCache &C, int device) {
  if (cudaSetDevice(device) != cudaSuccess) return GQM_ERR_NO_DEVICE;
  if (C.init) return GQM_OK;
  if (cudaStreamCreateWithFlags(&C.st, cudaStreamNonBlocking) != cudaSuccess) return GQM_ERR_CUDA;
  if (cudaEventCreate(&C.e0) != cudaSuccess || cudaEventCreate(&C.e1) != cudaSuccess) return GQM_ERR_CUDA;
  if (cudaMalloc((void **)&C.d_next, sizeof(int)) != cudaSuccess ||
      cudaMalloc((void **)&C.d_used, sizeof(unsigned long long)) != cudaSuccess)
    return GQM_ERR_MEMORY;
#ifndef GQM_HOST_EMU
  cudaDeviceGetAttribute(&C.sms, cudaDevAttrMultiProcessorCount, device);
#endif
  C.init = true;
  return GQM_OK;
}

int variant_of(const DevCache &C, const gqm_batch_options *b) {
  if (b && b->threads_per_block > 0) {
    for (int v = 0; v < kNumVariants; ++v)
      if (kVariants[v].threads == b->threads_per_block &&
          (b->blocks_per_sm <= 0 || kVariants[v].minb == b->blocks_per_sm))
        return v;
    return -1;
  }
  return C.tuned >= 0 ? C.tuned : kDefaultVariant;
}

// The whole call on one device: validation, the persistent launches (one per
// predicate mode present), then the single-domain path for domains that
// outgrew their arena.
int batch_call(int nd, const gqm_cdt_in *in, gqm_cdt_out *out, const gqm_options *opt, gqm_stats *stats,
               const gqm_batch_options *bopt, gqm_batch_report *rep, int *failed, int force_var, bool keep) {
  auto t0 = std::chrono::steady_clock::now();
  if (failed) *failed = -1;
  if (nd < 0 || (nd > 0 && (!in || !opt || (keep && !out)))) return GQM_ERR_ARGUMENT;
  if (rep) memset(rep, 0, sizeof(*rep));
  if (keep)
    for (int i = 0; i < nd; ++i) memset(&out[i], 0, sizeof(gqm_cdt_out));
  if (nd == 0) return GQM_OK;
  const int device = opt[0].device;
  if (device < 0 || device >= 16) return GQM_ERR_NO_DEVICE;
  for (int i = 0; i < nd; ++i) {
    int rc = check_domain(&in[i], &opt[i]);
    if (rc == GQM_OK && opt[i].device != device) rc = GQM_ERR_ARGUMENT;
    if (rc) {
      if (failed) *failed = i;
      return rc;
    }
  }
  DevCache &C = g_dev[device];
  std::lock_guard<std::mutex> lock(C.mu);
  int rc = setup_dev(C, device);
  if (rc) return rc;
  const int var = force_var >= 0 ? force_var : variant_of(C, bopt);
  if (var < 0) return GQM_ERR_ARGUMENT;
  const double frac = (bopt && bopt->memory_fraction > 0.0) ? bopt->memory_fraction : 0.8;
  std::vector<int> status(nd, GQM_ERR_CUDA);
  for (int pred = 0; pred < 2; ++pred) {
    std::vector<int> ids;
    for (int i = 0; i < nd; ++i)
      if ((opt[i].predicates ? 1 : 0) == pred) ids.push_back(i);
    rc = run_batch(C, ids, in, out, opt, stats, var, frac, status.data(), rep, keep);
    if (rc) {
      if (keep)
        for (int j = 0; j < nd; ++j) gqm_free_result(&out[j]);
      return rc;
    }
  }
  // domains that outgrew their arena: the single-domain path
  for (int i = 0; i < nd; ++i) {
    if (status[i] != GQM_ERR_ARENA) continue;
    if (rep) rep->fallbacks++;
    if (!keep) {
      status[i] = GQM_OK;
      continue;
    }
    gqm_stats st;
    status[i] = gqm_refine(&in[i], &out[i], &opt[i], &st);
    if (status[i] == GQM_OK && stats) stats[i] = st;
  }
  for (int i = 0; i < nd; ++i)
    if (status[i] != GQM_OK) {
      if (failed) *failed = i;
      if (keep)
        for (int j = 0; j < nd; ++j) gqm_free_result(&out[j]);
      return status[i];
    }
  if (rep) rep->total_ms = ms_since(t0);
  return GQM_OK;
}

}  // namespace
}  // namespace gqm

extern "C" {

void gqm_default_batch_options(gqm_batch_options *b) {
  if (!b) return;
  b->threads_per_block = 0;
  b->blocks_per_sm = 0;
  b->memory_fraction = 0.0;
}

int gqm_refine_batch_persistent(int ndomains, const gqm_cdt_in *in, gqm_cdt_out *out, const gqm_options *opt,
                                gqm_stats *stats, const gqm_batch_options *bopt, gqm_batch_report *report,
                                int *failed_domain) {
  return gqm::batch_call(ndomains, in, out, opt, stats, bopt, report, failed_domain, -1, true);
}

int gqm_batch_variants(int *threads, int *blocks_per_sm, int max) {
  for (int v = 0; v < gqm::kNumVariants && v < max; ++v) {
    if (threads) threads[v] = gqm::kVariants[v].threads;
    if (blocks_per_sm) blocks_per_sm[v] = gqm::kVariants[v].minb;
  }
  return gqm::kNumVariants;
}

int gqm_batch_autotune(int ndomains, const gqm_cdt_in *in, const gqm_options *opt, gqm_batch_options *chosen,
                       double *ms_per_variant) {
  if (ndomains <= 0 || !in || !opt) return GQM_ERR_ARGUMENT;
  int best = -1;
  double best_ms = 0.0;
  for (int v = 0; v < gqm::kNumVariants; ++v) {
    gqm_batch_report r;
    int failed = -1;
    int rc = gqm::batch_call(ndomains, in, nullptr, opt, nullptr, nullptr, &r, &failed, v, false);
    if (rc) return rc;
    if (ms_per_variant) ms_per_variant[v] = r.kernel_ms;
    if (best < 0 || r.kernel_ms < best_ms) {
      best = v;
      best_ms = r.kernel_ms;
    }
  }
  const int device = opt[0].device;
  {
    std::lock_guard<std::mutex> lock(gqm::g_dev[device].mu);
    gqm::g_dev[device].tuned = best;
  }
  if (chosen) {
    chosen->threads_per_block = gqm::kVariants[best].threads;
    chosen->blocks_per_sm = gqm::kVariants[best].minb;
    chosen->memory_fraction = 0.0;
  }
  return GQM_OK;
}

void gqm_batch_release(int device) {
  if (device < 0 || device >= 16) return;
  gqm::DevCache &C = gqm::g_dev[device];
  std::lock_guard<std::mutex> lock(C.mu);
  if (!C.init) return;
  cudaSetDevice(device);
  cudaStreamSynchronize(C.st);
  void *dev[] = {C.d_in, C.d_out, C.d_arena, C.d_jobs, C.d_order, C.d_next, C.d_used};
  for (void *p : dev)
    if (p) cudaFree(p);
  if (C.h_in) cudaFreeHost(C.h_in);
  if (C.h_out) cudaFreeHost(C.h_out);
  cudaEventDestroy(C.e0);
  cudaEventDestroy(C.e1);
  cudaStreamDestroy(C.st);
  const int tuned = C.tuned;
  C.d_in = C.d_out = C.d_arena = C.h_in = C.h_out = nullptr;
  C.in_cap = C.out_cap = C.arena_cap = C.h_in_cap = C.h_out_cap = 0;
  C.d_jobs = nullptr;
  C.d_order = nullptr;
  C.jobs_cap = 0;
  C.d_next = nullptr;
  C.d_used = nullptr;
  C.init = false;
  C.tuned = tuned;
}

}  // extern "C"
