// Constrained Delaunay triangulation on the GPU: the input construction step
// in front of the refiner.  Contract: Triangle's "pzQnc" (GPU_Refine/mesh.cpp:397,
// 220-239): zero-based, counterclockwise triangles, neighbour j opposite vertex
// j, every convex hull edge a segment.  All geometric decisions use exact
// predicates (predicates.h: floating-point filter, exact expansion fallback).
//
// Pipeline
//  1. Convex hull.  The extreme points in eight directions bound an octagon;
//     points strictly inside it are dropped on the device, the host runs the
//     monotone chain over the rest and keeps collinear hull points as
//     vertices (no input point may lie in the interior of a hull edge).
//  2. Initial triangulation: the hull polygon fanned around the non-hull point
//     nearest the hull's centroid.  Every other point finds its fan triangle by
//     an angular binary search.
//  3. Insertion rounds.  Each triangle holding pending points picks the one
//     with the smallest index.  A point strictly inside splits its triangle
//     1->3; a point on an edge splits both triangles of the edge 2->4.
//     Conflicts go to the smallest point index (64-bit claims whose high bits
//     carry a descending round stamp, so claims never need clearing); new
//     triangle slots are handed out by a prefix sum over the pending list, so
//     the numbering does not depend on thread timing.  Pending points move to
//     the child that contains them.  Lawson flips (edge-keyed claims) follow
//     every round until no edge is illegal.
//  4. Segments.  Edges already in the triangulation are marked.  Every missing
//     segment claims the channel of triangles it crosses; a segment holding
//     its whole channel recovers itself with Sloan's flip sequence inside the
//     channel, which only ever rewrites the channel's own slots.
//  5. Lawson flips of non-segment edges turn the result into the CDT.
//
// Neighbour words are oriented: (triangle << 2) | edge, -1 on the boundary.
// Every operation that rewrites triangles records, per old slot and edge, where
// that edge went (rmap); neighbours modified in the same launch fix their
// pointers through it in a second launch, unmodified neighbours are updated
// directly.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#ifndef GQM_HOST_EMU
#include <cub/device/device_scan.cuh>
#endif

#include "gqm_cdt.h"
#include "host_copy.h"
#include "predicates.h"

namespace gqm_cdt {

using u64 = unsigned long long;
constexpr int kNoSeg = 0x7fffffff;      // edge carries no segment
constexpr int kStampMax = 0x3fffffff;   // round stamps count up to this
constexpr int kThreads = 256;
constexpr int kMaxBlocks = 148 * 16;
// Kernels whose item count is only known on the device (flip rounds, pending
// points): one wave of four blocks per SM covers the grid-stride loop; idle
// rounds then cost one short wave instead of many.
constexpr int kWaveBlocks = 148 * 4;

#define CDEV __device__ __forceinline__
#define GRID_LOOP(i, n) \
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < (long)(n); i += (long)blockDim.x * gridDim.x)

CDEV int nx(int k) { return k == 2 ? 0 : k + 1; }
CDEV int pv(int k) { return k == 0 ? 2 : k - 1; }
CDEV int comp(const int4 &a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }
CDEV void setc(int4 &a, int k, int v) {
  if (k == 0)
    a.x = v;
  else if (k == 1)
    a.y = v;
  else
    a.z = v;
}
CDEV int get(const int4 *arr, long t, int k) { return reinterpret_cast<const int *>(arr + t)[k]; }
CDEV void put(int4 *arr, long t, int k, int v) { reinterpret_cast<int *>(arr + t)[k] = v; }
CDEV int4 i4(int a, int b, int c, int d) {
  int4 r;
  r.x = a;
  r.y = b;
  r.z = c;
  r.w = d;
  return r;
}
CDEV u64 stamp_hi(int stamp) { return (u64)(kStampMax - stamp) << 34; }
CDEV int sgn(double v) { return (v > 0) - (v < 0); }

// ---- predicates: the filters of predicates.h inline, exact tails out of line
__device__ __noinline__ double orient_tail(double ax, double ay, double bx, double by, double cx, double cy) {
  return gqm_orient_exact(ax, ay, bx, by, cx, cy);
}
CDEV double orient(double2 a, double2 b, double2 c) {
  double l = (a.x - c.x) * (b.y - c.y), r = (a.y - c.y) * (b.x - c.x), det = l - r;
  double bound = (3.0 + 16.0 * GQM_EPS) * GQM_EPS * (fabs(l) + fabs(r));
  if (det > bound || -det > bound) return det;
  return orient_tail(a.x, a.y, b.x, b.y, c.x, c.y);
}
__device__ __noinline__ double incircle_tail(double ax, double ay, double bx, double by, double cx, double cy,
                                             double dx, double dy) {
  return gqm_incircle_exact(ax, ay, bx, by, cx, cy, dx, dy);
}
// positive if d is strictly inside the circle through the counterclockwise a, b, c
CDEV double incircle(double2 a, double2 b, double2 c, double2 d) {
  double adx = a.x - d.x, bdx = b.x - d.x, cdx = c.x - d.x;
  double ady = a.y - d.y, bdy = b.y - d.y, cdy = c.y - d.y;
  double bdxcdy = bdx * cdy, cdxbdy = cdx * bdy, cdxady = cdx * ady, adxcdy = adx * cdy;
  double adxbdy = adx * bdy, bdxady = bdx * ady;
  double alift = adx * adx + ady * ady, blift = bdx * bdx + bdy * bdy, clift = cdx * cdx + cdy * cdy;
  double det = alift * (bdxcdy - cdxbdy) + blift * (cdxady - adxcdy) + clift * (adxbdy - bdxady);
  double perm = (fabs(bdxcdy) + fabs(cdxbdy)) * alift + (fabs(cdxady) + fabs(adxcdy)) * blift +
                (fabs(adxbdy) + fabs(bdxady)) * clift;
  double bound = (10.0 + 96.0 * GQM_EPS) * GQM_EPS * perm;
  if (det > bound || -det > bound) return det;
  return incircle_tail(a.x, a.y, b.x, b.y, c.x, c.y, d.x, d.y);
}
// a, b, c collinear: is c on the same side of a as b
CDEV bool same_dir(double2 a, double2 b, double2 c) {
  return sgn(b.x - a.x) == sgn(c.x - a.x) && sgn(b.y - a.y) == sgn(c.y - a.y);
}
CDEV unsigned fbits(float f) {
#ifdef GQM_HOST_EMU
  unsigned u;
  memcpy(&u, &f, 4);
  return u;
#else
  return __float_as_uint(f);
#endif
}

struct Dm {
  const double2 *P;
  int4 *tv, *tn, *tc;  // vertices, oriented neighbours, segment id per edge
  int4 *rmap, *rgeo;   // per rewritten slot: where each edge went; geometry for relocation
  u64 *claim, *pick;
  int *mst;            // stamp of the last round that rewrote the slot
  int *dst;            // tag of the dirty list that holds the slot
  int *loc;            // triangle holding a pending point, -1 once inserted
  int *err;
};

CDEV void set_err(int *err, int code) { atomicCAS(err, 0, code); }
// Slot in a list of length *len for every lane that wants one: one atomic
// per group of converged lanes, slots in lane order.  Every lane of the
// group calls it (want may be false).
CDEV int warp_slot(int *len, bool want) {
  unsigned m = __activemask();
  unsigned b = __ballot_sync(m, want);
  int lane = threadIdx.x & 31, leader = __ffs(m) - 1, base = 0;
  if (lane == leader && b) base = atomicAdd(len, __popc(b));
  base = __shfl_sync(m, base, leader);
  return base + __popc(b & ((1u << lane) - 1));
}
// Appends t to a dirty list unless it is there already (all lanes call it).
CDEV void dirty(const Dm &M, int t, bool want, int tag, int *list, int *cnt) {
  want = want && atomicExch(&M.dst[t], tag) != tag;
  int pos = warp_slot(cnt, want);
  if (want) list[pos] = t;
}
// back pointer of a neighbour that no operation of this round rewrites
CDEV void link_out(const Dm &M, int s, int e, int nb, int stamp) {
  if (nb >= 0 && M.mst[nb >> 2] != stamp) put(M.tn, nb >> 2, nb & 3, (s << 2) | e);
}
// pointer to a neighbour rewritten in this round: follow its edge map
CDEV void fix_edge(const Dm &M, int s, int e, int stamp) {
  int nb = get(M.tn, s, e);
  if (nb >= 0 && M.mst[nb >> 2] == stamp) put(M.tn, s, e, get(M.rmap, nb >> 2, nb & 3));
}

// ---------------------------------------------------------------------------
// hull and initial triangulation
// ---------------------------------------------------------------------------
__global__ void k_ext_partial(const double2 *P, int n, double *bv, int *bi) {
  double v[8];
  int id[8];
  for (int k = 0; k < 8; ++k) {
    v[k] = -INFINITY;
    id[k] = 0x7fffffff;
  }
  GRID_LOOP(i, n) {
    double2 p = P[i];
    double d[8] = {p.x, p.x + p.y, p.y, p.y - p.x, -p.x, -(p.x + p.y), -p.y, p.x - p.y};
    for (int k = 0; k < 8; ++k)
      if (d[k] > v[k]) {
        v[k] = d[k];
        id[k] = (int)i;
      }
  }
  __shared__ double sv[8][kThreads];
  __shared__ int si[8][kThreads];
  int tid = threadIdx.x;
  for (int k = 0; k < 8; ++k) {
    sv[k][tid] = v[k];
    si[k][tid] = id[k];
  }
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (tid < s)
      for (int k = 0; k < 8; ++k) {
        double ov = sv[k][tid + s];
        int oi = si[k][tid + s];
        if (ov > sv[k][tid] || (ov == sv[k][tid] && oi < si[k][tid])) {
          sv[k][tid] = ov;
          si[k][tid] = oi;
        }
      }
    __syncthreads();
  }
  if (tid == 0)
    for (int k = 0; k < 8; ++k) {
      bv[k * gridDim.x + blockIdx.x] = sv[k][0];
      bi[k * gridDim.x + blockIdx.x] = si[k][0];
    }
}

__global__ void k_ext_final(int nb, const double *bv, const int *bi, int *ext) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  for (int k = 0; k < 8; ++k) {
    double best = -INFINITY;
    int bidx = 0x7fffffff;
    for (int b = 0; b < nb; ++b) {
      double v = bv[k * nb + b];
      int i = bi[k * nb + b];
      if (v > best || (v == best && i < bidx)) {
        best = v;
        bidx = i;
      }
    }
    ext[k] = bidx == 0x7fffffff ? 0 : bidx;
  }
}

// Points not strictly inside the octagon of extreme points are hull candidates.
__global__ void k_oct_filter(const double2 *P, int n, const int *ext, int *cand, int *cnt) {
  int o[8], m = 0;
  for (int k = 0; k < 8; ++k)
    if (m == 0 || ext[k] != o[m - 1]) o[m++] = ext[k];
  while (m > 1 && o[m - 1] == o[0]) --m;
  GRID_LOOP(i, n) {
    double2 q = P[i];
    bool inside = m >= 3;
    for (int k = 0; k < m && inside; ++k) inside = orient(P[o[k]], P[o[k + 1 == m ? 0 : k + 1]], q) > 0;
    if (!inside) cand[atomicAdd(cnt, 1)] = (int)i;
  }
}

__global__ void k_fill(int *a, long n, int v) {
  GRID_LOOP(i, n) a[i] = v;
}
__global__ void k_mark_list(const int *list, int m, int *loc, int *hpos) {
  GRID_LOOP(i, m) {
    loc[list[i]] = -1;
    if (hpos) hpos[list[i]] = (int)i;
  }
}

// The non-hull point nearest (cx, cy): key = (float distance^2, index).
__global__ void k_center(const double2 *P, int n, const int *loc, double cx, double cy, u64 *best) {
  u64 b = ~0ull;
  GRID_LOOP(i, n) {
    if (loc[i] < 0) continue;
    double dx = P[i].x - cx, dy = P[i].y - cy;
    u64 key = ((u64)fbits((float)(dx * dx + dy * dy)) << 32) | (u64)i;
    if (key < b) b = key;
  }
  __shared__ u64 s[kThreads];
  int tid = threadIdx.x;
  s[tid] = b;
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if (tid < st && s[tid + st] < s[tid]) s[tid] = s[tid + st];
    __syncthreads();
  }
  if (tid == 0 && s[0] != ~0ull) atomicMin(best, s[0]);
}

// Fan T_i = (h_i, h_{i+1}, c) around the interior point c.
__global__ void k_fan(int H, const int *hull, int c, Dm M) {
  GRID_LOOP(i, H) {
    int t = (int)i, tnext = t + 1 == H ? 0 : t + 1, tprev = t == 0 ? H - 1 : t - 1;
    M.tv[t] = i4(hull[t], hull[tnext], c, 0);
    M.tn[t] = i4((tnext << 2) | 1, (tprev << 2) | 0, -1, 0);
    M.tc[t] = i4(kNoSeg, kNoSeg, kNoSeg, 0);
  }
}

CDEV int half_of(double2 c, double2 h0, double2 q) {
  double o = orient(c, h0, q);
  if (o > 0) return 0;
  if (o < 0) return 1;
  return same_dir(c, h0, q) ? 0 : 1;
}
// Fan triangle of every pending point: the last hull vertex whose angle around
// c (measured from h_0) does not exceed the point's.
__global__ void k_locate_fan(Dm M, int n, const int *hull, int H, int c) {
  double2 pc = M.P[c], h0 = M.P[hull[0]];
  GRID_LOOP(q, n) {
    if (M.loc[q] < 0) continue;
    double2 pq = M.P[q];
    int hq = half_of(pc, h0, pq);
    int lo = 0, hi = H - 1;
    while (lo < hi) {
      int mid = (lo + hi + 1) >> 1;
      double2 pm = M.P[hull[mid]];
      int hm = half_of(pc, h0, pm);
      bool le = hm != hq ? hm < hq : orient(pc, pm, pq) >= 0;
      if (le)
        lo = mid;
      else
        hi = mid - 1;
    }
    M.loc[q] = lo;
  }
}

// ---------------------------------------------------------------------------
// compaction helpers
// ---------------------------------------------------------------------------
__global__ void k_flag_pending(const int *pend, const int *pn, const int *loc, int *flag) {
  int n = *pn;
  GRID_LOOP(i, n) flag[i] = loc[pend[i]] >= 0;
}
__global__ void k_flag_all_pending(int n, const int *loc, int *flag) {
  GRID_LOOP(i, n) flag[i] = loc[i] >= 0;
}
__global__ void k_scatter(const int *src, int n, const int *flag, const int *rank, int *dst) {
  GRID_LOOP(i, n) {
    if (flag[i]) dst[rank[i]] = src ? src[i] : (int)i;
  }
}
__global__ void k_total(const int *flag, const int *rank, int n, int *out) {
  if (blockIdx.x == 0 && threadIdx.x == 0) *out = n > 0 ? rank[n - 1] + flag[n - 1] : 0;
}
__global__ void k_set(int *a, int v) {
  if (blockIdx.x == 0 && threadIdx.x == 0) *a = v;
}
__global__ void k_add(int *a, const int *b, int mul) {
  if (blockIdx.x == 0 && threadIdx.x == 0) *a += mul * *b;
}

// ---------------------------------------------------------------------------
// point insertion
// ---------------------------------------------------------------------------
__global__ void k_pick(Dm M, const int *pend, const int *pn, int stamp) {
  int n = *pn;
  u64 hi = stamp_hi(stamp);
  GRID_LOOP(i, n) {
    int q = pend[i];
    u64 key = hi | (u64)q, *pk = &M.pick[M.loc[q]];
    if (*pk > key) atomicMin(pk, key);  // most points of a crowded triangle see a smaller index already
  }
}

// ptype: -1 no insertion, 3 split 1->3, e in {0,1,2} split of edge e 2->4
__global__ void k_claim(Dm M, const int *pend, const int *pn, int stamp, int *ptype) {
  int n = *pn;
  u64 hi = stamp_hi(stamp);
  GRID_LOOP(i, n) {
    int q = pend[i], t = M.loc[q], ty = -1;
    u64 key = hi | (u64)q;
    if (M.pick[t] == key) {
      int4 v = M.tv[t];
      double2 p = M.P[q], a = M.P[v.x], b = M.P[v.y], c = M.P[v.z];
      if ((p.x == a.x && p.y == a.y) || (p.x == b.x && p.y == b.y) || (p.x == c.x && p.y == c.y)) {
        set_err(M.err, GQM_CDT_ERR_DUPLICATE);
      } else {
        double o0 = orient(b, c, p), o1 = orient(c, a, p), o2 = orient(a, b, p);
        if (o0 < 0 || o1 < 0 || o2 < 0) {
          set_err(M.err, GQM_CDT_ERR_INTERNAL);
        } else {
          int z = (o0 == 0) + (o1 == 0) + (o2 == 0);
          if (z == 0) {
            ty = 3;
            atomicMin(&M.claim[t], key);
          } else if (z == 1) {
            int e = o0 == 0 ? 0 : (o1 == 0 ? 1 : 2);
            int nb = get(M.tn, t, e);
            if (nb < 0) {
              set_err(M.err, GQM_CDT_ERR_INTERNAL);
            } else if (get(M.tc, t, e) != kNoSeg) {
              set_err(M.err, GQM_CDT_ERR_POINT_ON_SEGMENT);
            } else {
              ty = e;
              atomicMin(&M.claim[t], key);
              atomicMin(&M.claim[nb >> 2], key);
            }
          } else {
            set_err(M.err, GQM_CDT_ERR_DUPLICATE);
          }
        }
      }
    }
    ptype[i] = ty;
  }
}

__global__ void k_win_insert(Dm M, const int *pend, const int *pn, int stamp, const int *ptype, int *wflag) {
  int n = *pn;
  u64 hi = stamp_hi(stamp);
  GRID_LOOP(i, n) {
    int ty = ptype[i], ok = 0;
    if (ty >= 0) {
      int q = pend[i], t = M.loc[q];
      u64 key = hi | (u64)q;
      ok = M.claim[t] == key;
      int u = -1;
      if (ty < 3) {
        u = get(M.tn, t, ty) >> 2;
        ok = ok && M.claim[u] == key;
      }
      if (ok) {
        M.mst[t] = stamp;
        if (u >= 0) M.mst[u] = stamp;
      }
    }
    wflag[i] = ok;
  }
}

CDEV void split13(const Dm &M, int t, int q, int s1, int s2, int stamp) {
  int4 v = M.tv[t], n = M.tn[t], c = M.tc[t];
  M.tv[t] = i4(q, v.y, v.z, 0);
  M.tv[s1] = i4(v.x, q, v.z, 0);
  M.tv[s2] = i4(v.x, v.y, q, 0);
  M.tn[t] = i4(n.x, (s1 << 2) | 0, (s2 << 2) | 0, 0);
  M.tn[s1] = i4((t << 2) | 1, n.y, (s2 << 2) | 1, 0);
  M.tn[s2] = i4((t << 2) | 2, (s1 << 2) | 2, n.z, 0);
  M.tc[t] = i4(c.x, kNoSeg, kNoSeg, 0);
  M.tc[s1] = i4(kNoSeg, c.y, kNoSeg, 0);
  M.tc[s2] = i4(kNoSeg, kNoSeg, c.z, 0);
  M.rmap[t] = i4((t << 2) | 0, (s1 << 2) | 1, (s2 << 2) | 2, 3);
  M.rgeo[t] = i4(v.x, v.y, v.z, q);
  link_out(M, t, 0, n.x, stamp);
  link_out(M, s1, 1, n.y, stamp);
  link_out(M, s2, 2, n.z, stamp);
}

// q on edge i of t, shared with u (edge j).  t keeps v_{i+1} -> q, s1 takes
// v_{i+2} -> q; u keeps w_{j+1} -> q, s2 takes w_{j+2} -> q.
CDEV int split24(const Dm &M, int t, int i, int q, int s1, int s2, int stamp) {
  int4 v = M.tv[t], n = M.tn[t], c = M.tc[t];
  int nbr = comp(n, i), u = nbr >> 2, j = nbr & 3;
  int4 w = M.tv[u], m = M.tn[u], d = M.tc[u];
  int i1 = nx(i), i2 = nx(i1), j1 = nx(j), j2 = nx(j1);
  int ci = comp(c, i);
  int4 va = v, vb = v, wc = w, wd = w;
  setc(va, i1, q);
  setc(vb, i2, q);
  setc(wc, j1, q);
  setc(wd, j2, q);
  int4 na, nb, nc, nd, ca, cb, cc, cd;
  setc(na, i, (s2 << 2) | j);
  setc(na, i1, comp(n, i1));
  setc(na, i2, (s1 << 2) | i1);
  setc(nb, i, (u << 2) | j);
  setc(nb, i1, (t << 2) | i2);
  setc(nb, i2, comp(n, i2));
  setc(nc, j, (s1 << 2) | i);
  setc(nc, j1, comp(m, j1));
  setc(nc, j2, (s2 << 2) | j1);
  setc(nd, j, (t << 2) | i);
  setc(nd, j1, (u << 2) | j2);
  setc(nd, j2, comp(m, j2));
  setc(ca, i, ci);
  setc(ca, i1, comp(c, i1));
  setc(ca, i2, kNoSeg);
  setc(cb, i, ci);
  setc(cb, i1, kNoSeg);
  setc(cb, i2, comp(c, i2));
  setc(cc, j, ci);
  setc(cc, j1, comp(d, j1));
  setc(cc, j2, kNoSeg);
  setc(cd, j, ci);
  setc(cd, j1, kNoSeg);
  setc(cd, j2, comp(d, j2));
  na.w = nb.w = nc.w = nd.w = ca.w = cb.w = cc.w = cd.w = 0;
  M.tv[t] = va;
  M.tv[s1] = vb;
  M.tv[u] = wc;
  M.tv[s2] = wd;
  M.tn[t] = na;
  M.tn[s1] = nb;
  M.tn[u] = nc;
  M.tn[s2] = nd;
  M.tc[t] = ca;
  M.tc[s1] = cb;
  M.tc[u] = cc;
  M.tc[s2] = cd;
  int4 rt = i4(-1, -1, -1, 4 + i), ru = i4(-1, -1, -1, 4 + j);
  setc(rt, i1, (t << 2) | i1);
  setc(rt, i2, (s1 << 2) | i2);
  setc(ru, j1, (u << 2) | j1);
  setc(ru, j2, (s2 << 2) | j2);
  M.rmap[t] = rt;
  M.rmap[u] = ru;
  M.rgeo[t] = i4(v.x, v.y, v.z, q);
  M.rgeo[u] = i4(w.x, w.y, w.z, q);
  link_out(M, t, i1, comp(n, i1), stamp);
  link_out(M, s1, i2, comp(n, i2), stamp);
  link_out(M, u, j1, comp(m, j1), stamp);
  link_out(M, s2, j2, comp(m, j2), stamp);
  return u;
}

__global__ void k_split(Dm M, const int *pend, const int *pn, const int *ptype, const int *wflag, const int *wrank,
                        const int *ntri, int stamp, int tag, int *D, int *dcnt) {
  int n = *pn, nt0 = *ntri;
  GRID_LOOP(i, n) {
    bool win = wflag[i];
    int t = -1, u = -1, s1 = -1, s2 = -1;
    if (win) {
      int q = pend[i], ty = ptype[i];
      t = M.loc[q];
      s1 = nt0 + 2 * wrank[i];
      s2 = s1 + 1;
      M.loc[q] = -1;
      if (ty == 3)
        split13(M, t, q, s1, s2, stamp);
      else
        u = split24(M, t, ty, q, s1, s2, stamp);
    }
    // the children join the next flip round's list (no slot is in it yet)
    int pos = warp_slot(dcnt, win), pu = warp_slot(dcnt, u >= 0), p1 = warp_slot(dcnt, win),
        p2 = warp_slot(dcnt, win);
    if (win) {
      D[pos] = t;
      D[p1] = s1;
      D[p2] = s2;
      M.dst[t] = M.dst[s1] = M.dst[s2] = tag;
    }
    if (u >= 0) {
      D[pu] = u;
      M.dst[u] = tag;
    }
  }
}

__global__ void k_fix_insert(Dm M, const int *pend, const int *pn, const int *ptype, const int *wflag,
                             const int *wrank, const int *ntri, int stamp) {
  int n = *pn, nt0 = *ntri;
  GRID_LOOP(i, n) {
    if (!wflag[i]) continue;
    int ty = ptype[i];
    // the winner's point is inserted; its slot t is the child that kept it at index ty / 0
    int s1 = nt0 + 2 * wrank[i], s2 = s1 + 1;
    if (ty == 3) {
      int t = get(M.tn, s1, 0) >> 2;
      fix_edge(M, t, 0, stamp);
      fix_edge(M, s1, 1, stamp);
      fix_edge(M, s2, 2, stamp);
    } else {
      int i1 = nx(ty), i2 = nx(i1);
      int t = get(M.tn, s1, i1) >> 2;
      int nbu = get(M.tn, s1, ty), u = nbu >> 2, j = nbu & 3;
      fix_edge(M, t, i1, stamp);
      fix_edge(M, s1, i2, stamp);
      fix_edge(M, u, nx(j), stamp);
      fix_edge(M, s2, nx(nx(j)), stamp);
    }
  }
}

// Pending points find their triangle again once the flips of a round have
// converged: a visibility walk from the slot that held them (slots are reused
// in place, so it is nearby).  The triangulation is Delaunay at that point, so
// the walk cannot cycle; the step bound only guards the invariant.
__global__ void k_walk(Dm M, const int *pend, const int *pn) {
  int n = *pn;
  GRID_LOOP(i, n) {
    int q = pend[i], t = M.loc[q];
    double2 pq = M.P[q];
    for (int step = 0;; ++step) {
      if (step > (1 << 20)) {
        set_err(M.err, GQM_CDT_ERR_INTERNAL);
        break;
      }
      int4 v = M.tv[t];
      double2 a = M.P[v.x], b = M.P[v.y], c = M.P[v.z];
      int k = orient(b, c, pq) < 0 ? 0 : (orient(c, a, pq) < 0 ? 1 : (orient(a, b, pq) < 0 ? 2 : -1));
      if (k < 0) break;
      int nb = get(M.tn, t, k);
      if (nb < 0) {
        set_err(M.err, GQM_CDT_ERR_INTERNAL);
        break;
      }
      t = nb >> 2;
    }
    M.loc[q] = t;
  }
}

// ---------------------------------------------------------------------------
// Lawson flips
// ---------------------------------------------------------------------------
// Flips edge k of t (shared with u).  t = (x, y, z) with x opposite the edge,
// u = (w, z, y): afterwards t = (x, y, w) and u = (w, z, x).  With link set,
// unmodified outer neighbours get their back pointers here.
CDEV int flip(const Dm &M, int t, int k, int stamp, bool link) {
  int4 vt = M.tv[t], nt = M.tn[t], ct = M.tc[t];
  int k1 = nx(k), k2 = nx(k1);
  int x = comp(vt, k), y = comp(vt, k1), z = comp(vt, k2);
  int nbr = comp(nt, k), u = nbr >> 2, j = nbr & 3, j1 = nx(j), j2 = nx(j1);
  int4 vu = M.tv[u], nu = M.tn[u], cu = M.tc[u];
  int w = comp(vu, j);
  int A = comp(nt, k1), cA = comp(ct, k1), B = comp(nt, k2), cB = comp(ct, k2);
  int C = comp(nu, j1), cC = comp(cu, j1), D = comp(nu, j2), cD = comp(cu, j2);
  M.tv[t] = i4(x, y, w, 0);
  M.tn[t] = i4(C, (u << 2) | 1, B, 0);
  M.tc[t] = i4(cC, kNoSeg, cB, 0);
  M.tv[u] = i4(w, z, x, 0);
  M.tn[u] = i4(A, (t << 2) | 1, D, 0);
  M.tc[u] = i4(cA, kNoSeg, cD, 0);
  int4 rt = i4(-1, -1, -1, 8), ru = i4(-1, -1, -1, 8);
  setc(rt, k1, (u << 2) | 0);
  setc(rt, k2, (t << 2) | 2);
  setc(ru, j1, (t << 2) | 0);
  setc(ru, j2, (u << 2) | 2);
  M.rmap[t] = rt;
  M.rmap[u] = ru;
  M.rgeo[t] = M.rgeo[u] = i4(x, w, t, u);
  if (link) {
    link_out(M, t, 0, C, stamp);
    link_out(M, t, 2, B, stamp);
    link_out(M, u, 0, A, stamp);
    link_out(M, u, 2, D, stamp);
  }
  return u;
}

// Each edge of a dirty triangle that is not a segment and fails the incircle
// test claims its two triangles with key (stamp, t, k).  An edge between two
// dirty triangles is tested from the smaller one.  A triangle flipped in the
// previous round first fixes its outer pointers to neighbours that flipped in
// that round too (their edge maps are complete by now; the check of a
// triangle reads no other triangle's neighbour words).  Counters: dcur is
// this round's dirty count, dnext the next round's (cleared here for the
// apply launch).
__global__ void k_flip_check(Dm M, const int *D, const int *dcur, int *dnext, int tag, int stamp, int *C,
                             int *ccur) {
  int n = *dcur;
  if (blockIdx.x == 0 && threadIdx.x == 0) *dnext = 0;
  u64 hi = stamp_hi(stamp);
  GRID_LOOP(i, n) {
    int t = D[i];
    if (M.mst[t] == stamp - 1 && M.rmap[t].w == 8) {
      fix_edge(M, t, 0, stamp - 1);
      fix_edge(M, t, 2, stamp - 1);
    }
    int4 v = M.tv[t], nb = M.tn[t], c = M.tc[t];
    double2 a = M.P[v.x], b = M.P[v.y], cc3 = M.P[v.z];
    for (int k = 0; k < 3; ++k) {
      int e = comp(nb, k), u = e >> 2;
      bool bad = e >= 0 && comp(c, k) == kNoSeg && !(u < t && M.dst[u] == tag) &&
                 incircle(a, b, cc3, M.P[get(M.tv, u, e & 3)]) > 0;
      int code = (t << 2) | k;
      if (bad) {
        u64 key = hi | (u64)(unsigned)code;
        atomicMin(&M.claim[t], key);
        atomicMin(&M.claim[u], key);
      }
      int pos = warp_slot(ccur, bad);
      if (bad) C[pos] = code;
    }
  }
}

// ccur: this round's candidates; cnext: the next round's (cleared here)
__global__ void k_flip_win(Dm M, const int *C, const int *ccur, int *cnext, int stamp, int *wf) {
  int n = *ccur;
  if (blockIdx.x == 0 && threadIdx.x == 0) *cnext = 0;
  u64 hi = stamp_hi(stamp);
  GRID_LOOP(i, n) {
    int code = C[i], t = code >> 2, u = get(M.tn, t, code & 3) >> 2;
    u64 key = hi | (u64)(unsigned)code;
    int ok = M.claim[t] == key && M.claim[u] == key;
    wf[i] = ok;
    if (ok) M.mst[t] = M.mst[u] = stamp;
  }
}

__global__ void k_flip_apply(Dm M, const int *C, const int *ccur, const int *wf, int stamp, int tag, int *D,
                             int *dcnt, int *nflips) {
  int n = *ccur;
  GRID_LOOP(i, n) {
    int code = C[i], t = code >> 2, u = -1;
    bool win = wf[i];
    if (win) u = flip(M, t, code & 3, stamp, true);
    dirty(M, t, true, tag, D, dcnt);  // a loser is retried next round
    dirty(M, u, win, tag, D, dcnt);
    warp_slot(nflips, win);  // counts the flips
  }
}

__global__ void k_all_dirty(Dm M, int nt, int tag, int *D, int *dcnt) {
  GRID_LOOP(t, nt) dirty(M, (int)t, true, tag, D, dcnt);
}

// ---------------------------------------------------------------------------
// segments
// ---------------------------------------------------------------------------
__global__ void k_vt(Dm M, int nt, int *vt) {
  GRID_LOOP(t, nt) {
    int4 v = M.tv[t];
    vt[v.x] = (int)t;
    vt[v.y] = (int)t;
    vt[v.z] = (int)t;
  }
}

__global__ void k_seg_check(const int2 *S, int ns, int np, int *err) {
  GRID_LOOP(s, ns) {
    int2 e = S[s];
    if (e.x < 0 || e.y < 0 || e.x >= np || e.y >= np || e.x == e.y) set_err(err, GQM_CDT_ERR_SEGMENT);
  }
}

// Around vertex a: returns 1 with (*rt, *rk) the edge (a, b); 0 with *rt the
// triangle whose corner at a holds the direction to b and *rk the index of a
// in it; or an error code.
CDEV int star_find(const Dm &M, const int *vt, int a, int b, int *rt, int *rk) {
  int t0 = vt[a];
  double2 pa = M.P[a], pb = M.P[b];
  for (int dir = 0; dir < 2; ++dir) {
    int t = t0;
    for (int guard = 0; guard < (1 << 22); ++guard) {
      int4 v = M.tv[t];
      int ia = v.x == a ? 0 : (v.y == a ? 1 : (v.z == a ? 2 : -1));
      if (ia < 0) return GQM_CDT_ERR_INTERNAL;
      int y = comp(v, nx(ia)), z = comp(v, pv(ia));
      if (y == b) {
        *rt = t;
        *rk = pv(ia);
        return 1;
      }
      if (z == b) {
        *rt = t;
        *rk = nx(ia);
        return 1;
      }
      double2 py = M.P[y], pz = M.P[z];
      double oy = orient(pa, py, pb), oz = orient(pa, pz, pb);
      if ((oy == 0 && same_dir(pa, py, pb)) || (oz == 0 && same_dir(pa, pz, pb)))
        return GQM_CDT_ERR_POINT_ON_SEGMENT;
      if (oy > 0 && oz < 0) {
        *rt = t;
        *rk = ia;
        return 0;
      }
      int nb = get(M.tn, t, dir == 0 ? nx(ia) : pv(ia));
      if (nb < 0) break;
      t = nb >> 2;
      if (t == t0) return GQM_CDT_ERR_INTERNAL;
    }
  }
  return GQM_CDT_ERR_INTERNAL;
}

// Walks the triangles crossed by segment (a, b) from the corner (t, ia).
// Records the channel's triangles in R[0..m] and its crossed edges in Q[0..m)
// when given; returns m, the number of crossed edges, or an error code.
CDEV int walk(const Dm &M, int a, int b, int t, int ia, int cap, int *R, int2 *Q) {
  double2 pa = M.P[a], pb = M.P[b];
  int4 v = M.tv[t];
  int y = comp(v, nx(ia)), z = comp(v, pv(ia)), k = ia;
  if (R) R[0] = t;
  for (int m = 0; m < cap; ++m) {
    if (get(M.tc, t, k) != kNoSeg) return GQM_CDT_ERR_SEGMENTS_CROSS;
    int nb = get(M.tn, t, k);
    if (nb < 0) return GQM_CDT_ERR_INTERNAL;
    int u = nb >> 2, j = nb & 3, w = get(M.tv, u, j);
    if (R) {
      R[m + 1] = u;
      int2 e;
      e.x = y;
      e.y = z;
      Q[m] = e;
    }
    if (w == b) return m + 1;
    double o = orient(pa, pb, M.P[w]);
    if (o == 0) return GQM_CDT_ERR_POINT_ON_SEGMENT;
    if (o > 0) {
      z = w;
      k = nx(j);
    } else {
      y = w;
      k = pv(j);
    }
    t = u;
  }
  return GQM_CDT_ERR_INTERNAL;
}

CDEV void mark_edge(const Dm &M, int t, int k, int s) {
  atomicMin(reinterpret_cast<int *>(M.tc + t) + k, s);
  int nb = get(M.tn, t, k);
  if (nb >= 0) atomicMin(reinterpret_cast<int *>(M.tc + (nb >> 2)) + (nb & 3), s);
}

// Marks segments that are edges; lists the others.
__global__ void k_seg_mark(Dm M, const int *vt, const int2 *S, int ns, int *miss, int *mcnt) {
  GRID_LOOP(s, ns) {
    int2 e = S[s];
    int t, k;
    int r = star_find(M, vt, e.x, e.y, &t, &k);
    if (r < 0)
      set_err(M.err, r);
    else if (r == 1)
      mark_edge(M, t, k, (int)s);
    else
      miss[atomicAdd(mcnt, 1)] = (int)s;
  }
}

// Channel length (crossed edges) of every missing segment; -1 once the segment
// is an edge (then marked).
__global__ void k_chan_count(Dm M, const int *vt, const int2 *S, const int *miss, int nm, int cap, int *mlen,
                             int *sz) {
  GRID_LOOP(i, nm) {
    int s = miss[i];
    int2 e = S[s];
    int t, k, len = -1;
    int r = star_find(M, vt, e.x, e.y, &t, &k);
    if (r < 0) {
      set_err(M.err, r);
    } else if (r == 1) {
      mark_edge(M, t, k, s);
    } else {
      int m = walk(M, e.x, e.y, t, k, cap, nullptr, nullptr);
      if (m < 0)
        set_err(M.err, m);
      else
        len = m;
    }
    mlen[i] = len;
    sz[i] = len < 0 ? 0 : len + 4;
  }
}

__global__ void k_chan_claim(Dm M, const int *vt, const int2 *S, const int *miss, int nm, const int *mlen,
                             const int *off, int *R, int2 *Q, int stamp) {
  u64 hi = stamp_hi(stamp);
  GRID_LOOP(i, nm) {
    int m = mlen[i];
    if (m < 0) continue;
    int s = miss[i];
    int2 e = S[s];
    int t, k;
    star_find(M, vt, e.x, e.y, &t, &k);
    int *r = R + off[i];
    walk(M, e.x, e.y, t, k, m + 1, r, Q + off[i]);
    for (int j = 0; j <= m; ++j) atomicMin(&M.claim[r[j]], hi | (u64)s);
  }
}

__global__ void k_chan_win(Dm M, const int *miss, int nm, const int *mlen, const int *off, const int *R, int stamp,
                           int *wf) {
  u64 hi = stamp_hi(stamp);
  GRID_LOOP(i, nm) {
    int m = mlen[i], ok = m >= 0;
    u64 key = hi | (u64)miss[i];
    for (int j = 0; ok && j <= m; ++j) ok = M.claim[R[off[i] + j]] == key;
    if (ok)
      for (int j = 0; j <= m; ++j) M.mst[R[off[i] + j]] = stamp;
    wf[i] = ok;
  }
}

CDEV bool in_region(const Dm &M, int nb, u64 key) { return nb >= 0 && M.claim[nb >> 2] == key; }

// Flip inside a claimed channel: back pointers only for neighbours inside it.
CDEV void region_flip(const Dm &M, int t, int k, int stamp, u64 key) {
  int u = flip(M, t, k, stamp, false);
  int e;
  if (in_region(M, e = get(M.tn, t, 0), key)) put(M.tn, e >> 2, e & 3, (t << 2) | 0);
  if (in_region(M, e = get(M.tn, t, 2), key)) put(M.tn, e >> 2, e & 3, (t << 2) | 2);
  if (in_region(M, e = get(M.tn, u, 0), key)) put(M.tn, e >> 2, e & 3, (u << 2) | 0);
  if (in_region(M, e = get(M.tn, u, 2), key)) put(M.tn, e >> 2, e & 3, (u << 2) | 2);
}

CDEV bool find_edge(const Dm &M, const int *R, int nR, int p, int q, u64 key, bool outer, int *rt, int *rk) {
  for (int r = 0; r < nR; ++r) {
    int4 v = M.tv[R[r]];
    for (int k = 0; k < 3; ++k) {
      int y = comp(v, nx(k)), z = comp(v, pv(k));
      if (!((y == p && z == q) || (y == q && z == p))) continue;
      if (outer && in_region(M, get(M.tn, R[r], k), key)) continue;
      *rt = R[r];
      *rk = k;
      return true;
    }
  }
  return false;
}

// Sloan's edge recovery inside the channel of segment s = (a, b): crossed
// edges wait in a queue; a crossed edge whose quadrilateral is strictly convex
// is flipped and its replacement queued again while it still crosses the
// segment; a non-convex one goes to the back.  Flips only join triangles that
// share a crossed edge, so the channel's slots are the only ones rewritten.
__global__ void k_chan_sloan(Dm M, const int2 *S, const int *miss, int nm, const int *mlen, const int *off,
                             const int *R, int2 *Q, int4 *Bd, const int *wf, int stamp, int tag, int *D, int *dcnt,
                             int *nflips) {
  u64 hi = stamp_hi(stamp);
  GRID_LOOP(i, nm) {
    if (!wf[i]) continue;
    int s = miss[i], m = mlen[i], nR = m + 1;
    u64 key = hi | (u64)s;
    const int *reg = R + off[i];
    int2 *q = Q + off[i];
    int4 *bd = Bd + off[i];
    int a = S[s].x, b = S[s].y;
    double2 pa = M.P[a], pb = M.P[b];
    int nB = 0;
    for (int r = 0; r < nR; ++r) {
      int4 v = M.tv[reg[r]];
      for (int k = 0; k < 3; ++k)
        if (!in_region(M, get(M.tn, reg[r], k), key)) {
          if (nB < m + 3) bd[nB] = i4(reg[r], k, comp(v, nx(k)), comp(v, pv(k)));
          nB++;
        }
    }
    // m crossed edges; a vertex whose whole star the segment cuts adds an
    // uncrossed internal edge, so at most m + 3 edges face outside
    if (nB > m + 3) {
      set_err(M.err, GQM_CDT_ERR_INTERNAL);
      continue;
    }
    int head = 0, cnt = m, stall = 0, flips = 0, bad = 0;
    while (cnt > 0) {
      int2 e = q[head];
      head = head + 1 == m ? 0 : head + 1;
      cnt--;
      int t, k;
      if (!find_edge(M, reg, nR, e.x, e.y, key, false, &t, &k)) {
        bad = 1;
        break;
      }
      int nb = get(M.tn, t, k), u = nb >> 2;
      int x = get(M.tv, t, k), w = get(M.tv, u, nb & 3);
      int y = get(M.tv, t, nx(k)), z = get(M.tv, t, pv(k));
      double o1 = orient(M.P[x], M.P[w], M.P[y]), o2 = orient(M.P[x], M.P[w], M.P[z]);
      int tail = head + cnt >= m ? head + cnt - m : head + cnt;
      if (!((o1 > 0 && o2 < 0) || (o1 < 0 && o2 > 0))) {
        q[tail] = e;
        cnt++;
        if (++stall > cnt) {
          bad = 1;
          break;
        }
        continue;
      }
      stall = 0;
      region_flip(M, t, k, stamp, key);
      flips++;
      double ox = orient(pa, pb, M.P[x]), ow = orient(pa, pb, M.P[w]);
      if ((ox > 0 && ow < 0) || (ox < 0 && ow > 0)) {
        int2 ne;
        ne.x = x;
        ne.y = w;
        q[tail] = ne;
        cnt++;
      }
    }
    int t, k;
    if (bad || !find_edge(M, reg, nR, a, b, key, false, &t, &k)) {
      set_err(M.err, GQM_CDT_ERR_INTERNAL);
      continue;
    }
    put(M.tc, t, k, min(get(M.tc, t, k), s));
    int nb = get(M.tn, t, k);
    put(M.tc, nb >> 2, nb & 3, min(get(M.tc, nb >> 2, nb & 3), s));
    // where every boundary edge of the channel went
    for (int j = 0; j < nB; ++j) {
      int4 e = bd[j];
      int rt, rk;
      if (!find_edge(M, reg, nR, e.z, e.w, key, true, &rt, &rk)) {
        set_err(M.err, GQM_CDT_ERR_INTERNAL);
        break;
      }
      put(M.rmap, e.x, e.y, (rt << 2) | rk);
      link_out(M, rt, rk, get(M.tn, rt, rk), stamp);
    }
    for (int r = 0; r < nR; ++r)
      if (atomicExch(&M.dst[reg[r]], tag) != tag) D[atomicAdd(dcnt, 1)] = reg[r];
    atomicAdd(nflips, flips);
  }
}

__global__ void k_chan_fix(Dm M, const int *miss, int nm, const int *mlen, const int *off, const int *R,
                           const int *wf, int stamp) {
  u64 hi = stamp_hi(stamp);
  GRID_LOOP(i, nm) {
    if (!wf[i]) continue;
    u64 key = hi | (u64)miss[i];
    for (int r = 0; r <= mlen[i]; ++r) {
      int t = R[off[i] + r];
      for (int k = 0; k < 3; ++k) {
        int nb = get(M.tn, t, k);
        if (nb < 0 || M.claim[nb >> 2] == key) continue;
        if (M.mst[nb >> 2] == stamp) put(M.tn, t, k, get(M.rmap, nb >> 2, nb & 3));
      }
    }
  }
}

__global__ void k_chan_keep(const int *mlen, const int *wf, int nm, int *flag) {
  GRID_LOOP(i, nm) flag[i] = mlen[i] >= 0 && !wf[i];
}

// ---------------------------------------------------------------------------
// output
// ---------------------------------------------------------------------------
__global__ void k_out_tris(Dm M, int nt, int *tri, int *nbr) {
  GRID_LOOP(t, nt) {
    int4 v = M.tv[t], n = M.tn[t];
    tri[3 * t] = v.x;
    tri[3 * t + 1] = v.y;
    tri[3 * t + 2] = v.z;
    nbr[3 * t] = n.x < 0 ? -1 : n.x >> 2;
    nbr[3 * t + 1] = n.y < 0 ? -1 : n.y >> 2;
    nbr[3 * t + 2] = n.z < 0 ? -1 : n.z >> 2;
  }
}

// keep[s]: segment s is the first occurrence of its edge
__global__ void k_seg_keep(Dm M, const int *vt, const int2 *S, int ns, int *keep) {
  GRID_LOOP(s, ns) {
    int t, k, r = star_find(M, vt, S[s].x, S[s].y, &t, &k);
    if (r != 1) {
      set_err(M.err, r < 0 ? r : GQM_CDT_ERR_INTERNAL);
      keep[s] = 0;
    } else {
      keep[s] = get(M.tc, t, k) == (int)s;
    }
  }
}
__global__ void k_seg_out(const int2 *S, int ns, const int *keep, const int *rank, int2 *out) {
  GRID_LOOP(s, ns) {
    if (keep[s]) out[rank[s]] = S[s];
  }
}

// hflag[i] = 1 if hull edge (h_i, h_{i+1}) carries no input segment
__global__ void k_hull_flags(Dm M, int nt, const int *hpos, int *hflag) {
  GRID_LOOP(t, nt) {
    int4 v = M.tv[t], n = M.tn[t];
    for (int k = 0; k < 3; ++k)
      if (comp(n, k) < 0) hflag[hpos[comp(v, nx(k))]] = get(M.tc, t, k) == kNoSeg;
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
#ifdef GQM_HOST_EMU
#define KL(kernel, g, b) kernel
#else
#define KL(kernel, g, b) kernel<<<(g), (b), 0, st>>>
#endif

inline int grid_for(long n) {
  long g = (n + kThreads - 1) / kThreads;
  return (int)std::max(1L, std::min(g, (long)kMaxBlocks));
}

inline double host_orient(const double *P, int a, int b, int c) {
  return gqm_orient_exact(P[2 * a], P[2 * a + 1], P[2 * b], P[2 * b + 1], P[2 * c], P[2 * c + 1]);
}

// Monotone chain over the candidates, collinear boundary points kept, hull
// counterclockwise.  Returns 0, GQM_CDT_ERR_DUPLICATE or GQM_CDT_ERR_COLLINEAR.
int hull_chain(const double *P, std::vector<int> &cand, std::vector<int> &hull) {
  std::sort(cand.begin(), cand.end(), [&](int a, int b) {
    if (P[2 * a] != P[2 * b]) return P[2 * a] < P[2 * b];
    if (P[2 * a + 1] != P[2 * b + 1]) return P[2 * a + 1] < P[2 * b + 1];
    return a < b;
  });
  for (size_t i = 1; i < cand.size(); ++i)
    if (P[2 * cand[i]] == P[2 * cand[i - 1]] && P[2 * cand[i] + 1] == P[2 * cand[i - 1] + 1])
      return GQM_CDT_ERR_DUPLICATE;
  if (cand.size() < 3) return GQM_CDT_ERR_COLLINEAR;
  std::vector<int> L, U;
  for (int p : cand) {
    while (L.size() >= 2 && host_orient(P, L[L.size() - 2], L.back(), p) < 0) L.pop_back();
    L.push_back(p);
  }
  for (size_t i = cand.size(); i-- > 0;) {
    int p = cand[i];
    while (U.size() >= 2 && host_orient(P, U[U.size() - 2], U.back(), p) < 0) U.pop_back();
    U.push_back(p);
  }
  hull.assign(L.begin(), L.end() - 1);
  hull.insert(hull.end(), U.begin(), U.end() - 1);
  bool area = false;
  for (size_t k = 2; k < hull.size() && !area; ++k) area = host_orient(P, hull[0], hull[1], hull[k]) != 0;
  if (!area) return GQM_CDT_ERR_COLLINEAR;
  return 0;
}

// Triangulation of a convex polygon whose vertices may include collinear
// ones: clip a strict corner next to a flat vertex while flat vertices remain,
// any strict corner otherwise; no triangle is degenerate.
void clip_convex(const double *P, const std::vector<int> &h, std::vector<int> &tri) {
  int H = (int)h.size();
  std::vector<int> nxt(H), prv(H);
  for (int i = 0; i < H; ++i) {
    nxt[i] = (i + 1) % H;
    prv[i] = (i + H - 1) % H;
  }
  auto flat = [&](int i) { return host_orient(P, h[prv[i]], h[i], h[nxt[i]]) == 0; };
  std::vector<int> flats;
  for (int i = 0; i < H; ++i)
    if (flat(i)) flats.push_back(i);
  std::vector<char> gone(H, 0);
  int left = H, cur = 0;
  while (left > 3) {
    int g = -1;
    while (!flats.empty() && g < 0) {
      int f = flats.back();
      if (gone[f] || !flat(f)) {
        flats.pop_back();
        continue;
      }
      int a = nxt[f];
      while (flat(a)) a = nxt[a];
      g = a;
    }
    if (g < 0) {
      while (gone[cur]) cur = nxt[cur];
      g = cur;
    }
    tri.push_back(h[prv[g]]);
    tri.push_back(h[g]);
    tri.push_back(h[nxt[g]]);
    gone[g] = 1;
    nxt[prv[g]] = nxt[g];
    prv[nxt[g]] = prv[g];
    if (cur == g) cur = nxt[g];
    left--;
  }
  while (gone[cur]) cur = nxt[cur];
  tri.push_back(h[prv[cur]]);
  tri.push_back(h[cur]);
  tri.push_back(h[nxt[cur]]);
}

struct Builder {
  int dev = -1;
  cudaStream_t st = nullptr;
  long cap_np = 0, cap_ns = 0, cap_scratch = 0;
  // point / triangle buffers
  double2 *P = nullptr;
  int4 *tv = nullptr, *tn = nullptr, *tc = nullptr, *rmap = nullptr, *rgeo = nullptr;
  u64 *claim = nullptr, *pick = nullptr, *ubest = nullptr;
  int *mst = nullptr, *dst = nullptr, *loc = nullptr, *hpos = nullptr, *vt = nullptr;
  int *pend = nullptr, *pend2 = nullptr, *flag = nullptr, *rank = nullptr, *ptype = nullptr;
  int *D = nullptr, *D2 = nullptr, *C = nullptr, *wf = nullptr, *ctr = nullptr, *cand = nullptr, *hull = nullptr;
  double *bv = nullptr;
  int *bi = nullptr, *ext = nullptr;
  // segment buffers
  int2 *S = nullptr, *Sout = nullptr;
  int *miss = nullptr, *miss2 = nullptr, *mlen = nullptr, *msz = nullptr, *moff = nullptr, *keep = nullptr;
  int *R = nullptr;
  int2 *Q = nullptr;
  int4 *Bd = nullptr;
  int *out = nullptr;
  long out_cap = 0;
  void *cub_tmp = nullptr;
  size_t cub_bytes = 0;
  int *hc = nullptr;  // pinned counters
  int stamp = 0, tag = 0;
  long long launches = 0;

  // device counters in ctr[]
  // kNd and kNc hold two counters each (dirty list and candidates of
  // alternating flip rounds)
  enum { kErr = 0, kNtri, kNpend, kNd, kNc = kNd + 2, kFlips = kNc + 2, kTot, kMiss, kHcnt, kRecFlips, kNctr = 16 };

  template <class T>
  int dalloc(T **p, long n) {
    if (cudaMalloc((void **)p, sizeof(T) * (size_t)std::max(n, 1L)) != cudaSuccess) {
      *p = nullptr;
      return GQM_CDT_ERR_MEMORY;
    }
    return 0;
  }
  void free_all() {
    void *ps[] = {P, tv, tn, tc, rmap, rgeo, claim, pick, ubest, mst, dst, loc, hpos, vt, pend, pend2, flag,
                  rank, ptype, D, D2, C, wf, ctr, cand, hull, bv, bi, ext, S, Sout, miss, miss2, mlen, msz,
                  moff, keep, R, Q, Bd, out, cub_tmp};
    for (void *p : ps)
      if (p) cudaFree(p);
    P = nullptr;
    tv = tn = tc = rmap = rgeo = nullptr;
    claim = pick = ubest = nullptr;
    mst = dst = loc = hpos = vt = pend = pend2 = flag = rank = ptype = nullptr;
    D = D2 = C = wf = ctr = cand = hull = nullptr;
    bv = nullptr;
    bi = ext = nullptr;
    S = Sout = nullptr;
    miss = miss2 = mlen = msz = moff = keep = nullptr;
    R = nullptr;
    Q = nullptr;
    Bd = nullptr;
    out = nullptr;
    cub_tmp = nullptr;
    cap_np = cap_ns = cap_scratch = out_cap = 0;
    cub_bytes = 0;
  }
  void release() {
    free_all();
    if (hc) cudaFreeHost(hc);
    hc = nullptr;
    if (stage) cudaFreeHost(stage);
    stage = nullptr;
    stage_cap = 0;
    if (st) cudaStreamDestroy(st);
    st = nullptr;
    dev = -1;
  }

  int reserve(long np, long ns) {
    if (np <= cap_np && ns <= cap_ns) return 0;
    long n = std::max(np, cap_np), s = std::max(ns, cap_ns);
    free_all();
    long T = 2 * n + 8, nb = kMaxBlocks;
    int rc = 0;
    rc |= dalloc(&P, n);
    rc |= dalloc(&tv, T) | dalloc(&tn, T) | dalloc(&tc, T) | dalloc(&rmap, T) | dalloc(&rgeo, T);
    rc |= dalloc(&claim, T) | dalloc(&pick, T) | dalloc(&ubest, 1);
    rc |= dalloc(&mst, T) | dalloc(&dst, T) | dalloc(&loc, n) | dalloc(&hpos, n) | dalloc(&vt, n);
    rc |= dalloc(&pend, n) | dalloc(&pend2, n) | dalloc(&flag, std::max(n, s)) | dalloc(&rank, std::max(n, s));
    rc |= dalloc(&ptype, n) | dalloc(&D, T) | dalloc(&D2, T) | dalloc(&C, 3 * T) | dalloc(&wf, std::max(3 * T, s));
    rc |= dalloc(&ctr, kNctr) | dalloc(&cand, n) | dalloc(&hull, n) | dalloc(&bv, 8 * nb) | dalloc(&bi, 8 * nb);
    rc |= dalloc(&ext, 8);
    rc |= dalloc(&S, s) | dalloc(&Sout, s + n) | dalloc(&miss, s) | dalloc(&miss2, s) | dalloc(&mlen, s);
    rc |= dalloc(&msz, s) | dalloc(&moff, s) | dalloc(&keep, s);
    if (rc) return GQM_CDT_ERR_MEMORY;
#ifndef GQM_HOST_EMU
    size_t bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, bytes, (int *)nullptr, (int *)nullptr, (int)std::max(3 * T, s));
    if (cudaMalloc(&cub_tmp, bytes) != cudaSuccess) return GQM_CDT_ERR_MEMORY;
    cub_bytes = bytes;
#endif
    cap_np = n;
    cap_ns = s;
    // every slot starts with stamp 0 and tag 0; stamps and tags count up from 1 per call
    return 0;
  }
  int reserve_scratch(long n) {
    if (n <= cap_scratch) return 0;
    if (R) cudaFree(R);
    if (Q) cudaFree(Q);
    if (Bd) cudaFree(Bd);
    R = nullptr;
    Q = nullptr;
    Bd = nullptr;
    long c = std::max(n, 2 * cap_scratch);
    cap_scratch = 0;  // set again only once all three exist
    if (dalloc(&R, c) || dalloc(&Q, c) || dalloc(&Bd, c)) return GQM_CDT_ERR_MEMORY;
    cap_scratch = c;
    return 0;
  }

  void scan(const int *in, int *outp, int n) {
#ifdef GQM_HOST_EMU
    int s = 0;
    for (int i = 0; i < n; ++i) {
      int v = in[i];
      outp[i] = s;
      s += v;
    }
#else
    if (n > 0) cub::DeviceScan::ExclusiveSum(cub_tmp, cub_bytes, in, outp, n, st);
#endif
    launches += 1;
  }
  // counters to the host (one synchronisation)
  int sync_ctr() {
    cudaMemcpyAsync(hc, ctr, sizeof(int) * kNctr, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return GQM_CDT_ERR_CUDA;
    return hc[kErr];
  }
  Dm dm() {
    Dm M;
    M.P = P;
    M.tv = tv;
    M.tn = tn;
    M.tc = tc;
    M.rmap = rmap;
    M.rgeo = rgeo;
    M.claim = claim;
    M.pick = pick;
    M.mst = mst;
    M.dst = dst;
    M.loc = loc;
    M.err = ctr + kErr;
    return M;
  }

  // Lawson flips over the dirty list D (count in ctr[kNd], tag `tag`) until
  // no edge is illegal; three launches a round, one synchronisation every four
  // rounds.  Pending points then walk to their triangles.
  int lawson(int npend, gqm_cdt_gpu_stats *sts) {
    Dm M = dm();
    int *dbuf[2] = {D, D2};
    KL(k_set, 1, 1)(ctr + kNc, 0);
    launches++;
    int r = 0;
    for (int iter = 0;; ++iter) {
      for (int k = 0; k < 4; ++k, ++r) {
        ++stamp;
        int t2 = ++tag, p = r & 1, q = p ^ 1;
        KL(k_flip_check, kWaveBlocks, kThreads)(M, dbuf[p], ctr + kNd + p, ctr + kNd + q, tag - 1, stamp, C,
                                               ctr + kNc + p);
        KL(k_flip_win, kWaveBlocks, kThreads)(M, C, ctr + kNc + p, ctr + kNc + q, stamp, wf);
        KL(k_flip_apply, kWaveBlocks, kThreads)(M, C, ctr + kNc + p, wf, stamp, t2, dbuf[q], ctr + kNd + q,
                                               ctr + kFlips);
        launches += 3;
        if (sts) sts->flip_rounds++;
      }
      int e = sync_ctr();
      if (e) return e;
      if (hc[kNd + (r & 1)] == 0) break;
      if (iter > (1 << 20)) return GQM_CDT_ERR_INTERNAL;
    }
    if (npend > 0) {
      KL(k_walk, kWaveBlocks, kThreads)(M, pend, ctr + kNpend);
      launches++;
    }
    return 0;
  }

  // results of the last build (device arrays above)
  int n_pts = 0, n_tri = 0, n_seg = 0, last_status = 0;
  char *stage = nullptr;
  size_t stage_cap = 0;

  int build(int np, const double *pts, int ns, const int *segs, gqm_cdt_gpu_stats *sts);
  int download(gqm_cdt_result *res, gqm_cdt_gpu_stats *sts);
  int prepare(int device, int np, const double *pts, int ns, const int *segs, gqm_cdt_gpu_stats *sts);
};

#ifdef GQM_HOST_EMU
static Builder g_builder;
#else
static thread_local Builder g_builder;
#endif

using clk = std::chrono::steady_clock;
static double ms_since(clk::time_point t0) {
  return std::chrono::duration<double, std::milli>(clk::now() - t0).count();
}

int Builder::build(int np, const double *pts, int ns, const int *segs, gqm_cdt_gpu_stats *sts) {
  auto t_all = clk::now();
  if (np < 3) return GQM_CDT_ERR_FEW_POINTS;
  if (np > (1 << 28) || ns < 0 || ns > (1 << 29) || (ns > 0 && !segs)) return GQM_CDT_ERR_SEGMENT;
  int rc = reserve(np, ns);
  if (rc) return rc;
  // mst starts at 0 for every slot, so no stamp - 1 seen by a flip check may be
  // 0: stamps start at 1 (edge maps left by an earlier build are never read)
  stamp = 1;
  tag = 0;
  launches = 0;
  long T = 2L * np + 8;
  cudaMemsetAsync(ctr, 0, sizeof(int) * kNctr, st);
  cudaMemsetAsync(mst, 0, sizeof(int) * T, st);
  cudaMemsetAsync(dst, 0, sizeof(int) * T, st);
  cudaMemsetAsync(claim, 0xff, sizeof(u64) * T, st);
  cudaMemsetAsync(pick, 0xff, sizeof(u64) * T, st);
  auto t0 = clk::now();
  cudaMemcpyAsync(P, pts, sizeof(double) * 2 * (size_t)np, cudaMemcpyHostToDevice, st);
  if (ns) cudaMemcpyAsync(S, segs, sizeof(int) * 2 * (size_t)ns, cudaMemcpyHostToDevice, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) return GQM_CDT_ERR_CUDA;
  if (sts) sts->ms_h2d = ms_since(t0);
  Dm M = dm();

  // 1. hull
  t0 = clk::now();
#ifdef GQM_HOST_EMU
  int nb = 1;  // one emulated block covers the grid
#else
  int nb = std::min(grid_for(np), 2 * 148);  // the final reduction runs on one thread
#endif
  KL(k_ext_partial, nb, kThreads)(P, np, bv, bi);
  KL(k_ext_final, 1, 1)(nb, bv, bi, ext);
  KL(k_oct_filter, grid_for(np), kThreads)(P, np, ext, cand, ctr + kHcnt);
  if (ns) KL(k_seg_check, grid_for(ns), kThreads)(S, ns, np, ctr + kErr);
  launches += 3 + (ns > 0);
  if ((rc = sync_ctr())) return rc;
  int nc = hc[kHcnt];
  std::vector<int> hcand(nc), hl;
  cudaMemcpyAsync(hcand.data(), cand, sizeof(int) * (size_t)nc, cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) return GQM_CDT_ERR_CUDA;
  if ((rc = hull_chain(pts, hcand, hl))) return rc;
  int H = (int)hl.size();
  if (sts) {
    sts->hull_candidates = nc;
    sts->hull_vertices = H;
  }
  cudaMemcpyAsync(hull, hl.data(), sizeof(int) * H, cudaMemcpyHostToDevice, st);
  KL(k_fill, grid_for(np), kThreads)(loc, np, 0);
  KL(k_fill, grid_for(np), kThreads)(hpos, np, -1);
  KL(k_mark_list, grid_for(H), kThreads)(hull, H, loc, hpos);
  launches += 3;
  int ntri;
  int npend = 0;
  if (H < np) {
    double cx = 0, cy = 0;
    for (int h : hl) {
      cx += pts[2 * h];
      cy += pts[2 * h + 1];
    }
    cx /= H;
    cy /= H;
    cudaMemsetAsync(ubest, 0xff, sizeof(u64), st);
    KL(k_center, grid_for(np), kThreads)(P, np, loc, cx, cy, ubest);
    u64 hb;
    cudaMemcpyAsync(&hb, ubest, sizeof(u64), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return GQM_CDT_ERR_CUDA;
    int c = (int)(hb & 0xffffffffu);
    if (hb == ~0ull || c < 0 || c >= np) return GQM_CDT_ERR_INTERNAL;
    int cl[1] = {c};
    cudaMemcpyAsync(flag, cl, sizeof(int), cudaMemcpyHostToDevice, st);
    KL(k_mark_list, 1, kThreads)(flag, 1, loc, nullptr);
    KL(k_fan, grid_for(H), kThreads)(H, hull, c, M);
    KL(k_locate_fan, grid_for(np), kThreads)(M, np, hull, H, c);
    ntri = H;
    // pending list in index order
    KL(k_flag_all_pending, grid_for(np), kThreads)(np, loc, flag);
    scan(flag, rank, np);
    KL(k_scatter, grid_for(np), kThreads)(nullptr, np, flag, rank, pend);
    KL(k_total, 1, 1)(flag, rank, np, ctr + kNpend);
    launches += 7;
    npend = np - H - 1;
  } else {
    std::vector<int> tri;
    clip_convex(pts, hl, tri);
    ntri = (int)tri.size() / 3;
    // adjacency by matching edges (the polygon is small)
    std::vector<int4> htv(ntri), htn(ntri), htc(ntri);
    std::vector<std::pair<uint64_t, int>> ek;
    for (int t = 0; t < ntri; ++t) {
      htv[t] = int4{tri[3 * t], tri[3 * t + 1], tri[3 * t + 2], 0};
      htn[t] = int4{-1, -1, -1, 0};
      htc[t] = int4{kNoSeg, kNoSeg, kNoSeg, 0};
      for (int k = 0; k < 3; ++k) {
        uint32_t a = (uint32_t)tri[3 * t + (k + 1) % 3], b = (uint32_t)tri[3 * t + (k + 2) % 3];
        ek.push_back({((uint64_t)std::min(a, b) << 32) | std::max(a, b), (t << 2) | k});
      }
    }
    std::sort(ek.begin(), ek.end());
    for (size_t i = 1; i < ek.size(); ++i)
      if (ek[i].first == ek[i - 1].first) {
        int x = ek[i].second, y = ek[i - 1].second;
        (&htn[x >> 2].x)[x & 3] = y;
        (&htn[y >> 2].x)[y & 3] = x;
      }
    cudaMemcpyAsync(tv, htv.data(), sizeof(int4) * ntri, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(tn, htn.data(), sizeof(int4) * ntri, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(tc, htc.data(), sizeof(int4) * ntri, cudaMemcpyHostToDevice, st);
    KL(k_set, 1, 1)(ctr + kNpend, 0);
    launches++;
  }
  KL(k_set, 1, 1)(ctr + kNtri, ntri);
  // the initial triangulation is not Delaunay: every triangle starts dirty
  ++tag;
  KL(k_set, 1, 1)(ctr + kNd, 0);
  KL(k_all_dirty, grid_for(ntri), kThreads)(M, ntri, tag, D, ctr + kNd);
  launches += 3;
  if ((rc = lawson(npend, sts))) return rc;
  if (sts) sts->ms_hull = ms_since(t0);

  // 2. insertion rounds
  t0 = clk::now();
  while (npend > 0) {
    ++stamp;
    int t2 = ++tag;
    KL(k_pick, kMaxBlocks, kThreads)(M, pend, ctr + kNpend, stamp);
    KL(k_claim, kMaxBlocks, kThreads)(M, pend, ctr + kNpend, stamp, ptype);
    KL(k_win_insert, kMaxBlocks, kThreads)(M, pend, ctr + kNpend, stamp, ptype, flag);
    scan(flag, rank, npend);
    KL(k_set, 1, 1)(ctr + kNd, 0);
    KL(k_split, kMaxBlocks, kThreads)(M, pend, ctr + kNpend, ptype, flag, rank, ctr + kNtri, stamp, t2, D,
                                      ctr + kNd);
    KL(k_fix_insert, kMaxBlocks, kThreads)(M, pend, ctr + kNpend, ptype, flag, rank, ctr + kNtri, stamp);
    KL(k_total, 1, 1)(flag, rank, npend, ctr + kTot);
    KL(k_add, 1, 1)(ctr + kNtri, ctr + kTot, 2);
    // drop inserted points from the pending list (order kept)
    KL(k_flag_pending, kMaxBlocks, kThreads)(pend, ctr + kNpend, loc, flag);
    scan(flag, rank, npend);
    KL(k_scatter, grid_for(npend), kThreads)(pend, npend, flag, rank, pend2);
    KL(k_total, 1, 1)(flag, rank, npend, ctr + kNpend);
    std::swap(pend, pend2);
    launches += 11;
    if (sts) sts->insert_rounds++;
    if ((rc = sync_ctr())) return rc;
    if (hc[kTot] == 0) return GQM_CDT_ERR_INTERNAL;  // no progress
    npend = hc[kNpend];
    if ((rc = lawson(npend, sts))) return rc;
  }
  if ((rc = sync_ctr())) return rc;
  ntri = hc[kNtri];
  if (ntri != 2 * np - H - 2) return GQM_CDT_ERR_INTERNAL;
  if (sts) {
    sts->flips = hc[kFlips];
    sts->ms_insert = ms_since(t0);
  }

  // 3. segments
  t0 = clk::now();
  if (ns > 0) {
    KL(k_vt, grid_for(ntri), kThreads)(M, ntri, vt);
    KL(k_seg_mark, grid_for(ns), kThreads)(M, vt, S, ns, miss, ctr + kMiss);
    launches += 2;
    if ((rc = sync_ctr())) return rc;
    int nm = hc[kMiss];
    if (sts) sts->segments_missing = nm;
    ++tag;  // the dirty list of the final flips collects every rewritten channel
    int acc_tag = tag;
    KL(k_set, 1, 1)(ctr + kNd, 0);
    launches++;
    int rounds = 0;
    while (nm > 0) {
      if (++rounds > 100000) return GQM_CDT_ERR_INTERNAL;
      ++stamp;
      KL(k_chan_count, grid_for(nm), kThreads)(M, vt, S, miss, nm, ntri, mlen, msz);
      scan(msz, moff, nm);
      KL(k_total, 1, 1)(msz, moff, nm, ctr + kTot);
      launches += 2;
      if ((rc = sync_ctr())) return rc;
      if ((rc = reserve_scratch(std::max(hc[kTot], 1)))) return rc;
      KL(k_chan_claim, grid_for(nm), kThreads)(M, vt, S, miss, nm, mlen, moff, R, Q, stamp);
      KL(k_chan_win, grid_for(nm), kThreads)(M, miss, nm, mlen, moff, R, stamp, wf);
      KL(k_chan_sloan, grid_for(nm), kThreads)(M, S, miss, nm, mlen, moff, R, Q, Bd, wf, stamp, acc_tag, D,
                                               ctr + kNd, ctr + kRecFlips);
      KL(k_chan_fix, grid_for(nm), kThreads)(M, miss, nm, mlen, moff, R, wf, stamp);
      KL(k_chan_keep, grid_for(nm), kThreads)(mlen, wf, nm, flag);
      scan(flag, rank, nm);
      KL(k_scatter, grid_for(nm), kThreads)(miss, nm, flag, rank, miss2);
      KL(k_total, 1, 1)(flag, rank, nm, ctr + kMiss);
      KL(k_vt, grid_for(ntri), kThreads)(M, ntri, vt);
      std::swap(miss, miss2);
      launches += 8;
      if ((rc = sync_ctr())) return rc;
      nm = hc[kMiss];
    }
    if (sts) {
      sts->recover_rounds = rounds;
      sts->recover_flips = hc[kRecFlips];
    }
    long long before = hc[kFlips];
    ++stamp;  // channel slots carry flip maps of this phase; the first check must not read them
    if ((rc = lawson(0, sts))) return rc;
    if (sts) sts->flips += hc[kFlips] - before;
  }
  if (sts) sts->ms_segments = ms_since(t0);

  // 4. output on the device: triangles, neighbours (plain indices), the kept
  // input segments, then the hull edges that carry none
  t0 = clk::now();
  long need = 6L * ntri;
  if (need > out_cap) {
    if (out) cudaFree(out);
    out = nullptr;
    out_cap = 0;
    if (dalloc(&out, need)) return GQM_CDT_ERR_MEMORY;
    out_cap = need;
  }
  KL(k_out_tris, grid_for(ntri), kThreads)(M, ntri, out, out + 3L * ntri);
  KL(k_vt, grid_for(ntri), kThreads)(M, ntri, vt);
  KL(k_set, 1, 1)(ctr + kTot, 0);
  launches += 3;
  if (ns > 0) {
    KL(k_seg_keep, grid_for(ns), kThreads)(M, vt, S, ns, keep);
    scan(keep, rank, ns);
    KL(k_seg_out, grid_for(ns), kThreads)(S, ns, keep, rank, Sout);
    KL(k_total, 1, 1)(keep, rank, ns, ctr + kTot);
    launches += 3;
  }
  KL(k_fill, grid_for(H), kThreads)(flag, H, 0);
  KL(k_hull_flags, grid_for(ntri), kThreads)(M, ntri, hpos, flag);
  launches += 2;
  if ((rc = sync_ctr())) return rc;
  int nkeep = hc[kTot];
  std::vector<int> hflag(H);
  cudaMemcpyAsync(hflag.data(), flag, sizeof(int) * H, cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) return GQM_CDT_ERR_CUDA;
  std::vector<int2> hseg;
  for (int i = 0; i < H; ++i)
    if (hflag[i]) {
      int2 e;
      e.x = hl[i];
      e.y = hl[(i + 1) % H];
      hseg.push_back(e);
    }
  if (!hseg.empty())
    cudaMemcpyAsync(Sout + nkeep, hseg.data(), sizeof(int2) * hseg.size(), cudaMemcpyHostToDevice, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) return GQM_CDT_ERR_CUDA;
  n_pts = np;
  n_tri = ntri;
  n_seg = nkeep + (int)hseg.size();
  if (sts) {
    sts->ms_output = ms_since(t0);
    sts->kernel_launches = launches;
    sts->ms_total = ms_since(t_all);
  }
  return 0;
}

// The result of the last build, from the device into malloc'ed arrays: one
// copy into pinned staging, then the host's cores split it up.
int Builder::download(gqm_cdt_result *res, gqm_cdt_gpu_stats *sts) {
  auto t0 = clk::now();
  size_t bt = sizeof(int) * 3 * (size_t)n_tri, bs = sizeof(int) * 2 * (size_t)n_seg;
  size_t bytes = 2 * bt + bs;
  if (bytes > stage_cap) {
    if (stage) cudaFreeHost(stage);
    stage = nullptr;
    stage_cap = 0;
    if (cudaMallocHost((void **)&stage, bytes) != cudaSuccess) return GQM_CDT_ERR_MEMORY;
    stage_cap = bytes;
  }
  cudaMemcpyAsync(stage, out, 2 * bt, cudaMemcpyDeviceToHost, st);
  if (bs) cudaMemcpyAsync(stage + 2 * bt, Sout, bs, cudaMemcpyDeviceToHost, st);
  res->numberofpoints = n_pts;
  res->numberoftriangles = n_tri;
  res->numberofsegments = n_seg;
  res->trianglelist = (int *)malloc(bt + 8);
  res->neighborlist = (int *)malloc(bt + 8);
  res->segmentlist = (int *)malloc(bs + 8);
  if (!res->trianglelist || !res->neighborlist || !res->segmentlist) return GQM_CDT_ERR_MEMORY;
  advise_huge(res->trianglelist, bt);
  advise_huge(res->neighborlist, bt);
  if (cudaStreamSynchronize(st) != cudaSuccess) return GQM_CDT_ERR_CUDA;
  host_copy({{res->trianglelist, stage, bt}, {res->neighborlist, stage + bt, bt}, {res->segmentlist, stage + 2 * bt, bs}});
  if (sts) {
    sts->ms_d2h = ms_since(t0);
    sts->ms_total += sts->ms_d2h;
  }
  return 0;
}

// Points and segments in; the refiner's device input out (arrays owned by the builder).
int Builder::prepare(int device, int np, const double *pts, int ns, const int *segs, gqm_cdt_gpu_stats *stats) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
    return last_status = GQM_CDT_ERR_NO_DEVICE;
  if (dev != device) {
    release();
    if (cudaSetDevice(device) != cudaSuccess) return GQM_CDT_ERR_NO_DEVICE;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return GQM_CDT_ERR_CUDA;
    if (cudaMallocHost((void **)&hc, sizeof(int) * kNctr) != cudaSuccess) return GQM_CDT_ERR_MEMORY;
    dev = device;
  } else if (cudaSetDevice(device) != cudaSuccess) {
    return GQM_CDT_ERR_NO_DEVICE;
  }
  if (!pts && np > 0) return last_status = GQM_CDT_ERR_FEW_POINTS;
  int rc = build(np, pts, ns, segs, stats);
  last_status = rc;
  if (rc && (rc == GQM_CDT_ERR_CUDA || cudaGetLastError() != cudaSuccess)) release();
  return rc;
}

}  // namespace gqm_cdt

extern "C" {

int gqm_cdt_build_gpu(int np, const double *pts, int ns, const int *segs, int device, gqm_cdt_result *out,
                      gqm_cdt_gpu_stats *stats) {
  using namespace gqm_cdt;
  if (!out) return GQM_CDT_ERR_INTERNAL;
  memset(out, 0, sizeof(*out));
  if (stats) memset(stats, 0, sizeof(*stats));
  Builder &B = g_builder;
  int rc = B.prepare(device, np, pts, ns, segs, stats);
  if (rc == 0) rc = B.download(out, stats);
  if (rc) {
    free(out->trianglelist);
    free(out->neighborlist);
    free(out->segmentlist);
    memset(out, 0, sizeof(*out));
  }
  return out->status = rc;
}

int gqm_triangulate_refine(int np, const double *pts, int ns, const int *segs, const gqm_options *opt,
                           gqm_cdt_out *out, gqm_stats *stats, gqm_cdt_gpu_stats *cdt_stats) {
  using namespace gqm_cdt;
  if (!out || !opt) return GQM_ERR_ARGUMENT;
  memset(out, 0, sizeof(*out));
  if (cdt_stats) memset(cdt_stats, 0, sizeof(*cdt_stats));
  if (opt->device < 0 || opt->device >= 64) return GQM_ERR_NO_DEVICE;
  Builder &B = g_builder;
  int rc = B.prepare(opt->device, np, pts, ns, segs, cdt_stats);
  if (rc) return GQM_ERR_INPUT_CDT;
  // one refiner context per device, kept between calls
  static std::mutex m;
  static gqm_context *ctx[64] = {};
  std::lock_guard<std::mutex> lock(m);
  if (!ctx[opt->device] && (rc = gqm_context_create(opt->device, &ctx[opt->device]))) return rc;
  gqm_cdt_in in;
  in.numberofpoints = B.n_pts;
  in.pointlist = reinterpret_cast<const double *>(B.P);
  in.numberoftriangles = B.n_tri;
  in.trianglelist = B.out;
  in.neighborlist = B.out + 3L * B.n_tri;
  in.numberofsegments = B.n_seg;
  in.segmentlist = reinterpret_cast<const int *>(B.Sout);
  rc = gqm_context_run(ctx[opt->device], &in, 1, opt, stats);
  if (rc == GQM_OK) rc = gqm_context_result(ctx[opt->device], out);
  return rc;
}

int gqm_cdt_gpu_last_status(void) { return gqm_cdt::g_builder.last_status; }

void gqm_cdt_gpu_free(gqm_cdt_result *r) {
  if (!r) return;
  free(r->trianglelist);
  free(r->neighborlist);
  free(r->segmentlist);
  memset(r, 0, sizeof(*r));
}

void gqm_cdt_gpu_release(void) { gqm_cdt::g_builder.release(); }

}  // extern "C"
