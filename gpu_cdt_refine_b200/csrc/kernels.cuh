// Kernels of the B200 refiner.  Each kernel restates one step of the
// reference's GPU pipeline (GPU_Refine/refine.cu; the line ranges are cited at
// every kernel) over the structure-of-arrays mesh of gqm_device.cuh.  Kernels
// are grid-stride loops whose element count is read from device memory, so a
// launch never waits for the host to learn a count.
#pragma once
#include "gqm_device.cuh"
#include "learned.cuh"

// Register budget of the latency-bound walk kernels (flip checks, cavity
// walks, link updates): ask for at least this many resident 256-thread blocks
// per SM, so enough warps are in flight to cover their dependent loads.
#ifndef GQM_WALK_MIN_BLOCKS
#define GQM_WALK_MIN_BLOCKS 2
#endif

// Three compilations of the same kernels:
//  * grid mode (default): every step below is a __global__ kernel whose
//    grid-stride loop covers its items across the whole grid;
//  * CTA mode (GQM_CTA_MODE, batch.cu): every step is a __device__ function
//    that one thread block runs over one domain's items, the block's threads
//    striding over them; the caller separates steps with __syncthreads();
//  * cluster mode (GQM_CLUSTER_MODE, flipcl.cu): every step is a __device__
//    function that the blocks of one thread-block cluster (the whole grid of
//    the launch) run together, striding over the items with all their
//    threads; the caller separates steps with cluster barriers.
#if defined(GQM_CTA_MODE)
#define GQM_KERNEL __device__
#define GQM_WALK_BOUNDS
#define GQM_BOUNDS(minb)
#define GQM_GTID ((int)threadIdx.x)
#define GQM_GSIZE ((int)blockDim.x)
#define GQM_BLOCK0 true
#elif defined(GQM_CLUSTER_MODE)
#define GQM_KERNEL __device__
#define GQM_WALK_BOUNDS
#define GQM_BOUNDS(minb)
#define GQM_GTID ((int)(blockIdx.x * blockDim.x + threadIdx.x))
#define GQM_GSIZE ((int)(gridDim.x * blockDim.x))
#define GQM_BLOCK0 (blockIdx.x == 0)
#else
#define GQM_KERNEL __global__
#define GQM_WALK_BOUNDS __launch_bounds__(256, GQM_WALK_MIN_BLOCKS)
#define GQM_BOUNDS(minb) __launch_bounds__(256, minb)
#define GQM_GTID ((int)(blockIdx.x * blockDim.x + threadIdx.x))
#define GQM_GSIZE ((int)(gridDim.x * blockDim.x))
#define GQM_BLOCK0 (blockIdx.x == 0)
#endif

namespace gqm {

#define GS_LOOP(i, n) for (int i = GQM_GTID; i < (n); i += GQM_GSIZE)

// Counts and slot lists that some kernels take either as values (the
// block-mode engine, whose driver holds them in registers) or as device words
// that an earlier kernel of the same CUDA graph wrote (the single-domain
// engine, whose driver state lives on the device).
struct DevInt {
  const int *p;
};
__device__ __forceinline__ int nval(int n) { return n; }
__device__ __forceinline__ int nval(DevInt d) { return *d.p; }
// free slots handed out from base[*off] on
struct DevSlots {
  const int *base;
  const int *off;
};
__device__ __forceinline__ const int *slots_of(const int *p) { return p; }
__device__ __forceinline__ const int *slots_of(DevSlots s) { return s.base + *s.off; }

// ============================================================================
// Initialisation (refine.cu:5557-5747, 3105-3151)
// ============================================================================

// findIncidentOri (refine.cu:35-93): edge index, in neighbour n, of the edge
// shared with t; -1 when they do not share two vertices.
__device__ __forceinline__ int incident_ori(const int *tri, int t, int n) {
  if (t < 0 || n < 0) return -1;
  int inc0 = -1, inc1 = -1, count = 0;
  for (int i = 0; i < 3; i++) {
    int a = tri[3 * t + i];
    for (int j = 0; j < 3; j++)
      if (a == tri[3 * n + j]) {
        if (count == 0) {
          inc0 = j;
          count = 1;
          continue;
        }
        inc1 = j;
        break;
      }
  }
  if (inc0 == -1 || inc1 == -1) return -1;
  int d = inc0 - inc1;
  int idx = (d == -1 || d == 2) ? inc0 : inc1;
  return idx == 0 ? 2 : (idx == 1 ? 0 : 1);
}

// Input index check, run before anything dereferences the input: vertices in
// [0, np), neighbours in [-1, nt), segment endpoints in [0, np) and distinct,
// coordinates finite.  The reference trusts its input; a bad index here would
// make the initialisation read outside the input arrays.
GQM_KERNEL void k_check_input(const double2 *pts, int np, const int *tri, const int *nbr, int nt,
                              const int *seg, int ns, int *err) {
  int bad = 0;
  GS_LOOP(i, np) {
    double2 p = pts[i];
    if (!isfinite(p.x) || !isfinite(p.y)) bad = 1;
  }
  GS_LOOP(t, nt) {
    for (int k = 0; k < 3; k++) {
      unsigned v = (unsigned)tri[3 * t + k];
      int n = nbr[3 * t + k];
      if (v >= (unsigned)np || n < -1 || n >= nt) bad = 1;
    }
  }
  GS_LOOP(s, ns) {
    unsigned a = (unsigned)seg[2 * s], b = (unsigned)seg[2 * s + 1];
    if (a >= (unsigned)np || b >= (unsigned)np || a == b) bad = 1;
  }
  if (bad) atomicCAS(err, 0, GQM_ERR_ARGUMENT);
}

GQM_KERNEL void k_init_tris(Mesh M, const int *tri, const int *nbr, int nt, int tcap) {
  GS_LOOP(t, tcap) {
    if (t < nt) {
      M.tv[t] = make_int4(tri[3 * t], tri[3 * t + 1], tri[3 * t + 2], 0);
      int4 nb;
      nb.x = etri(nbr[3 * t], incident_ori(tri, t, nbr[3 * t]));
      nb.y = etri(nbr[3 * t + 1], incident_ori(tri, t, nbr[3 * t + 1]));
      nb.z = etri(nbr[3 * t + 2], incident_ori(tri, t, nbr[3 * t + 2]));
      nb.w = 0;
      M.tn[t] = nb;
      M.tst[t] = TS_NOTNULL | TS_CHECK;
    } else {
      M.tv[t] = make_int4(0, 0, 0, 0);
      M.tn[t] = make_int4(0, 0, 0, 0);
      M.tst[t] = 0;
    }
    M.tsg[t] = make_int4(-1, -1, -1, 0);
    M.tflip[t] = 0;
    M.tfo[t] = 0;
    M.tmark[t] = 0;
    M.tpos[t] = -1;
  }
}

GQM_KERNEL void k_init_points(Mesh M, const double2 *pts, int np, int pcap) {
  GS_LOOP(i, pcap) {
    if (i < np) {
      M.pts[i] = pts[i];
      M.ps[i] = 0;
    } else {
      M.pts[i] = make_double2(0.0, 0.0);
      M.ps[i] = PS_DELETED;
    }
    M.pred[i] = 0;
  }
}

// cos^2(theta) exactly as the reference evaluates it on the device
// (refine.cu:418, 123-124).
#define GQM_PI 3.141592653589793238462643383279502884197169399375105820974944592308
GQM_KERNEL void k_goodcos(double theta, double *out) {
  if (threadIdx.x == 0 && GQM_BLOCK0) {
    double c = cos(theta * GQM_PI / 180.0);
    out[0] = c * c;
    out[1] = cos(theta * GQM_PI / 180.0) * cos(theta * GQM_PI / 180.0);
  }
}

__device__ __forceinline__ unsigned long long seg_key(int a, int b) {
  unsigned lo = (unsigned)min(a, b), hi = (unsigned)max(a, b);
  return ((unsigned long long)hi << 32) | lo;
}
__device__ __forceinline__ unsigned seg_hash(unsigned long long k, unsigned mask) {
  return (unsigned)((k * 0x9E3779B97F4A7C15ull) >> 24) & mask;
}
GQM_KERNEL void k_seg_hash_insert(const int2 *segs, int ns, unsigned long long *keys, int *vals, unsigned mask) {
  GS_LOOP(s, ns) {
    unsigned long long k = seg_key(segs[s].x, segs[s].y);
    unsigned h = seg_hash(k, mask);
    for (unsigned probe = 0; probe <= mask; ++probe) {
      unsigned long long old = atomicCAS(keys + h, ~0ull, k);
      if (old == ~0ull) {
        vals[h] = s;
        break;
      }
      h = (h + 1) & mask;
    }
  }
}
// initSubsegs (refine.cu:5618-5747) for every triangle: edge (p0,p1) is
// orientation 2, (p1,p2) 0, (p2,p0) 1; subseg2tri keeps the largest otri
// (atomicMax), tri2subseg the largest matching subsegment.
GQM_KERNEL void k_init_subsegs(Mesh M, int nt, const unsigned long long *keys, const int *vals, unsigned mask,
                               int *s2t_int) {
  GS_LOOP(t, nt) {
    int4 v = M.tv[t];
    int4 sg = make_int4(-1, -1, -1, 0);
    const int eu[3] = {v.x, v.y, v.z}, ew[3] = {v.y, v.z, v.x}, eo[3] = {2, 0, 1};
    for (int e = 0; e < 3; ++e) {
      unsigned long long k = seg_key(eu[e], ew[e]);
      unsigned h = seg_hash(k, mask);
      for (unsigned probe = 0; probe <= mask; ++probe) {
        unsigned long long kk = keys[h];
        if (kk == ~0ull) break;
        if (kk == k) {
          int s = vals[h];
          atomicMax(s2t_int + s, (t << 2) | eo[e]);
          if (s > comp(sg, eo[e])) setc(sg, eo[e], s);
        }
        h = (h + 1) & mask;
      }
    }
    M.tsg[t] = sg;
  }
}
GQM_KERNEL void k_pack_s2t(Mesh M, const int *s2t_int, int ns) {
  GS_LOOP(s, ns) {
    M.s2t[s] = s2t_plain(s2t_int[s]);
    M.s2seg[s] = s;
  }
}

// kernelMarkAllEncsegs, refine.cu:3105-3151
template <class N>
GQM_KERNEL void k_mark_all_encsegs(Mesh M, N ns_) {
  const int ns = nval(ns_);
  GS_LOOP(s, ns) {
    int e = -1;
    int otri = s2t_get(M, s);
    if (otri >= 0) {
      int t = dtri(otri), o = dori(otri);
      int4 v = M.tv[t];
      double2 vo = M.pts[comp(v, m3(o + 1))], vd = M.pts[comp(v, m3(o + 2))], va = M.pts[comp(v, o)];
      if (encroached(vo, vd, va, M.gc2, M.mode)) e = 0;
      int on = ld1(M.tn, t, o);
      if (on != -1) {
        double2 vb = M.pts[ld1(M.tv, dtri(on), dori(on))];
        if (encroached(vd, vo, vb, M.gc2, M.mode)) e = 0;
      }
    }
    M.enc[s] = e;
  }
}

// ============================================================================
// Bad triangles (refine.cu:317-497)
// ============================================================================
// kernelComputeSmallestAngle, refine.cu:317-374: cos^2 of the smallest angle
__device__ __forceinline__ double smallest_cos2(double2 pA, double2 pO, double2 pD, int *shortest) {
  double dxod = pO.x - pD.x, dyod = pO.y - pD.y;
  double dxda = pD.x - pA.x, dyda = pD.y - pA.y;
  double dxao = pA.x - pO.x, dyao = pA.y - pO.y;
  // gqm_madd: the products the reference's contracted build fuses (see
  // predicates.h); the sums are the same in either order
  double lenOrg = gqm_madd(dyod, dyod, dxod * dxod);
  double lenDest = gqm_madd(dyda, dyda, dxda * dxda);
  double lenApex = gqm_madd(dxao, dxao, dyao * dyao);
  double ang, sh;
  if (lenOrg < lenDest && lenOrg < lenApex) {
    sh = lenOrg;
    *shortest = 0;
    ang = gqm_madd(dyda, dyao, dxda * dxao);
  } else if (lenDest < lenOrg && lenDest < lenApex) {
    sh = lenDest;
    *shortest = 1;
    ang = gqm_madd(dyod, dyao, dxod * dxao);
  } else {
    sh = lenApex;
    *shortest = 2;
    ang = gqm_madd(dyod, dyda, dxod * dxda);
  }
  return ang * ang * sh / (lenOrg * lenDest * lenApex);
}

// kernelMarkBadTriangles, refine.cu:376-497, over every triangle slot below
// ntri that is not null and has CHECK set.
template <class N>
GQM_KERNEL void k_mark_bad(Mesh M, N ntri_) {
  const int ntri = nval(ntri_);
  GS_LOOP(t, ntri) {
    uint8_t st = M.tst[t];
    if (!(st & TS_NOTNULL) || !(st & TS_CHECK)) continue;
    st = (uint8_t)((st & ~TS_CHECK) | TS_NOTNULL);
    int4 v = M.tv[t];
    double2 a = M.pts[v.x], b = M.pts[v.y], c = M.pts[v.z];
    int sh;
    double c2 = smallest_cos2(a, b, c, &sh);
    bool bad = true;
    if (c2 <= M.gc2) {
      bad = false;
    } else if (ld1(M.tsg, t, sh) == -1) {
      int eOrg = comp(v, m3(sh + 1)), eDest = comp(v, m3(sh + 2));
      if ((M.ps[eOrg] & PS_SEGSPLIT) && (M.ps[eDest] & PS_SEGSPLIT)) {
        int s1 = -1, s2 = -1;
        int cur = t, ori = sh, guard = 0;
        do {
          int o = ld1(M.tn, cur, ori);
          cur = dtri(o);
          ori = m3(dori(o) + 1);
          if (cur < 0 || ++guard > (1 << 20)) break;
          s1 = ld1(M.tsg, cur, ori);
        } while (s1 == -1);
        cur = t;
        ori = sh;
        guard = 0;
        do {
          int o = ld1(M.tn, cur, ori);
          cur = dtri(o);
          ori = m3(dori(o) + 2);
          if (cur < 0 || ++guard > (1 << 20)) break;
          s2 = ld1(M.tsg, cur, ori);
        } while (s2 == -1);
        if (s1 < 0 || s2 < 0) {
          raise_err(M, -5);
        } else {
          int2 g1 = M.segs[M.s2seg[s1]], g2 = M.segs[M.s2seg[s2]];
          int common = -1;
          if (g1.x == g2.x || g1.x == g2.y)
            common = g1.x;
          else if (g1.y == g2.x || g1.y == g2.y)
            common = g1.y;
          if (common != -1) {
            double2 vo = (sh == 0) ? b : (sh == 1 ? c : a);
            double2 vd = (sh == 0) ? c : (sh == 1 ? a : b);
            double2 vc = M.pts[common];
            double d1 = gqm_madd(vc.x - vo.x, vc.x - vo.x, (vc.y - vo.y) * (vc.y - vo.y));
            double d2 = gqm_madd(vc.x - vd.x, vc.x - vd.x, (vc.y - vd.y) * (vc.y - vd.y));
            if ((d1 < 1.001 * d2) && (d1 > 0.999 * d2)) bad = false;
          }
        }
      }
    }
    // area bound (no counterpart in the reference; Triangle's `a` switch)
    if (!bad && M.max_area > 0.0 &&
        0.5 * fabs((b.x - a.x) * (c.y - a.y) - (b.y - a.y) * (c.x - a.x)) > M.max_area)
      bad = true;
    M.tst[t] = bad ? (uint8_t)(st | TS_BAD) : (uint8_t)(st & ~TS_BAD);
  }
}

// ============================================================================
// Flip-flop (refine.cu:580-2490)
// ============================================================================
// markFan, refine.cu:580-602
__device__ void mark_fan(const Mesh &M, int triIndex, int triOri) {
  int cur = triIndex, ori = triOri, guard = 0;
  do {
    M.tflip[cur] = 1;
    int nx = ld1(M.tn, cur, m3(ori + 2));
    cur = dtri(nx);
    ori = dori(nx);
    if (++guard > (1 << 20)) {
      raise_err(M, -4);
      return;
    }
  } while (cur > -1 && cur != triIndex);
}

__device__ __forceinline__ bool is_red(const Mesh &M, int p) { return M.pred[p] != 0; }

// Direction of a 4-2 flip, recomputed from the partner's current vertices
// (refine.cu:1232-1250, 1740-1758, 2120-2138).
__device__ __forceinline__ bool flip42_outward(const Mesh &M, int pOppTri, int pOppOri) {
  int4 q = M.tv[pOppTri];
  int mn = kMaxInt;
  if (is_red(M, q.x) && q.x < mn) mn = q.x;
  if (is_red(M, q.y) && q.y < mn) mn = q.y;
  if (is_red(M, q.z) && q.z < mn) mn = q.z;
  return mn == comp(q, m3(pOppOri + 2));
}

// kernelInitLinklist, refine.cu:1172-1278.  Besides the winner's triangle
// list, each listed triangle records its list slot in tpos so that phase 2
// finds it directly instead of by binary search over the winners.
__device__ void init_link_body(const Mesh &M, int pos, int index, int *ll) {
  {
    int ori = M.tfo[index];
    int l[4] = {index, -1, -1, -1};
    if (ori < 3) {
      l[1] = dtri(ld1(M.tn, index, m3(ori + 1)));
    } else if (ori < 6) {
      ori = m3(ori - 3 + 1);
      l[1] = dtri(ld1(M.tn, index, ori));
      l[2] = dtri(ld1(M.tn, index, m3(ori + 2)));
    } else {
      ori -= 6;
      int pOpp = ld1(M.tn, index, ori);
      int pOppTri = dtri(pOpp), pOppOri = dori(pOpp);
      bool outward = flip42_outward(M, pOppTri, pOppOri);
      l[1] = pOppTri;
      if (outward) {
        l[2] = dtri(ld1(M.tn, index, m3(ori + 2)));
        l[3] = dtri(ld1(M.tn, pOppTri, m3(pOppOri + 1)));
      } else {
        l[2] = dtri(ld1(M.tn, index, m3(ori + 1)));
        l[3] = dtri(ld1(M.tn, pOppTri, m3(pOppOri + 2)));
      }
    }
    for (int k = 0; k < 4; ++k) {
      ll[4 * pos + k] = l[k];
      if (l[k] >= 0) M.tpos[l[k]] = 4 * pos + k;
    }
  }
}

__device__ __forceinline__ void set_tri(const Mesh &M, int a, int b, int c, int t, int ori) {
  int4 v;
  setc(v, m3(ori + 1), a);
  setc(v, m3(ori + 2), b);
  setc(v, ori, c);
  v.w = 0;
  M.tv[t] = v;
}
__device__ __forceinline__ void set_link(int *sl, int nOrg, int nDest, int nApex, int li, int ori) {
  sl[li * 3 + ori] = nOrg;
  sl[li * 3 + m3(ori + 1)] = nDest;
  sl[li * 3 + m3(ori + 2)] = nApex;
}

// kernelUpdatePhase1, refine.cu:1295-1552
// The subseg2tri stores are not made here but collected in `ps` (their key
// needs the winner's position in the reference's list, found afterwards).
struct PendingS2T {
  int n;
  int s[6], v[6], slot[6];
  __device__ __forceinline__ void add(int sg, int val, int sl) {
    s[n] = sg;
    v[n] = val;
    slot[n] = sl;
    n++;
  }
};
__device__ void phase1_body(const Mesh &M, int pos, int index, int *sl, PendingS2T &ps) {
  {
    int ori = M.tfo[index];
    if (ori < 3) {
      int pOpp = ld1(M.tn, index, m3(ori + 1));
      int pOppTri = dtri(pOpp), pOppOri = dori(pOpp);
      int4 vi = M.tv[index], vp = M.tv[pOppTri];
      int4 ni = M.tn[index], np = M.tn[pOppTri];
      int4 si = M.tsg[index], sp = M.tsg[pOppTri];
      int pOrg = comp(vi, m3(ori + 1)), pDest = comp(vi, m3(ori + 2)), pApex = comp(vi, ori);
      int pO = comp(vp, pOppOri);
      int nOrg = comp(ni, ori), nApex = comp(ni, m3(ori + 2));
      int npDest = comp(np, m3(pOppOri + 1)), npApex = comp(np, m3(pOppOri + 2));
      set_tri(M, pOrg, pDest, pO, index, ori);
      set_tri(M, pApex, pOrg, pO, pOppTri, pOppOri);
      set_link(sl, nOrg + 3, kMaxInt, nApex + 3, 4 * pos, ori);
      set_link(sl, kMaxInt, npDest + 3, npApex + 3, 4 * pos + 1, pOppOri);
      int sOrg = comp(si, ori), sApex = comp(si, m3(ori + 2));
      int spDest = comp(sp, m3(pOppOri + 1)), spApex = comp(sp, m3(pOppOri + 2));
      int4 a, b;
      setc(a, ori, sOrg);
      setc(a, m3(ori + 1), spDest);
      setc(a, m3(ori + 2), -1);
      a.w = 0;
      setc(b, pOppOri, sApex);
      setc(b, m3(pOppOri + 2), spApex);
      setc(b, m3(pOppOri + 1), -1);
      b.w = 0;
      M.tsg[index] = a;
      M.tsg[pOppTri] = b;
      if (sOrg != -1) ps.add(sOrg, (index << 2) | ori, 0);
      if (spDest != -1) ps.add(spDest, (index << 2) | m3(ori + 1), 1);
      if (sApex != -1) ps.add(sApex, (pOppTri << 2) | pOppOri, 2);
      if (spApex != -1) ps.add(spApex, (pOppTri << 2) | m3(pOppOri + 2), 3);
      M.tst[index] |= TS_CHECK;
      M.tst[pOppTri] |= TS_CHECK;
    } else if (ori < 6) {
      ori = m3(ori - 3 + 1);
      int t1 = ld1(M.tn, index, ori), t2 = ld1(M.tn, index, m3(ori + 2));
      int t1_ori = dori(t1), t2_ori = dori(t2);
      t1 = dtri(t1);
      t2 = dtri(t2);
      int4 vi = M.tv[index];
      int pOrg = comp(vi, m3(ori + 1)), pDest = comp(vi, m3(ori + 2)), pApex = comp(vi, ori);
      M.ps[pOrg] |= PS_DELETED;
      pOrg = ld1(M.tv, t1, t1_ori);
      int nOrg = ld1(M.tn, t1, m3(t1_ori + 2)), nDest = ld1(M.tn, index, m3(ori + 1));
      int nApex = ld1(M.tn, t2, m3(t2_ori + 1));
      set_tri(M, pOrg, pDest, pApex, index, ori);
      set_link(sl, nOrg + 3, nDest + 3, nApex + 3, 4 * pos, ori);
      sl[(4 * pos + 1) * 3 + m3(t1_ori + 2)] = nOrg + 3;
      sl[(4 * pos + 2) * 3 + m3(t2_ori + 1)] = nApex + 3;
      int sOrg = ld1(M.tsg, index, m3(ori + 1)), sApex = ld1(M.tsg, t1, m3(t1_ori + 2));
      int sDest = ld1(M.tsg, t2, m3(t2_ori + 1));
      int4 a;
      setc(a, m3(ori + 1), sOrg);
      setc(a, ori, sApex);
      setc(a, m3(ori + 2), sDest);
      a.w = 0;
      M.tsg[index] = a;
      if (sOrg != -1) ps.add(sOrg, (index << 2) | m3(ori + 1), 4);
      if (sApex != -1) ps.add(sApex, (index << 2) | ori, 5);
      if (sDest != -1) ps.add(sDest, (index << 2) | m3(ori + 2), 6);
      M.tst[index] |= TS_CHECK;
      M.tst[t1] &= (uint8_t)~TS_NOTNULL;
      M.tst[t2] &= (uint8_t)~TS_NOTNULL;
    } else {
      ori -= 6;
      int pOpp = ld1(M.tn, index, ori);
      int pOppTri = dtri(pOpp), pOppOri = dori(pOpp);
      int4 vi = M.tv[index];
      int pOrg = comp(vi, m3(ori + 1)), pDest = comp(vi, m3(ori + 2)), pApex = comp(vi, ori);
      int pO = ld1(M.tv, pOppTri, pOppOri);
      bool outw = is_red(M, pOrg) && (!is_red(M, pDest) || pOrg < pDest);
      int t1, t2;
      if (outw) {
        t1 = ld1(M.tn, index, m3(ori + 2));
        t2 = ld1(M.tn, pOppTri, m3(pOppOri + 1));
      } else {
        t1 = ld1(M.tn, index, m3(ori + 1));
        t2 = ld1(M.tn, pOppTri, m3(pOppOri + 2));
      }
      int t1_ori = dori(t1), t2_ori = dori(t2);
      t1 = dtri(t1);
      t2 = dtri(t2);
      int nOpp = ld1(M.tv, t1, t1_ori);
      int sOrg, sDest, sApex, snOrg, snDest, snApex;
      if (outw) {
        M.ps[pOrg] |= PS_DELETED;
        int nOrg = ld1(M.tn, pOppTri, m3(pOppOri + 2)), nDest = ld1(M.tn, index, m3(ori + 1));
        int npDest = ld1(M.tn, t1, m3(t1_ori + 1)), npApex = ld1(M.tn, t2, m3(t2_ori + 2));
        set_tri(M, pO, pDest, pApex, index, ori);
        set_tri(M, pO, pApex, nOpp, t1, t1_ori);
        set_link(sl, nOrg + 3, nDest + 3, kMaxInt, 4 * pos, ori);
        set_link(sl, kMaxInt, npDest + 3, npApex + 3, 4 * pos + 2, t1_ori);
        sl[(4 * pos + 1) * 3 + m3(pOppOri + 2)] = nOrg + 3;
        sl[(4 * pos + 3) * 3 + m3(t2_ori + 2)] = npApex + 3;
        sOrg = ld1(M.tsg, pOppTri, m3(pOppOri + 2));
        sDest = ld1(M.tsg, index, m3(ori + 1));
        sApex = ld1(M.tsg, index, m3(ori + 2));
        snOrg = ld1(M.tsg, t1, t1_ori);
        snDest = ld1(M.tsg, t1, m3(t1_ori + 1));
        snApex = ld1(M.tsg, t2, m3(t2_ori + 2));
      } else {
        M.ps[pDest] |= PS_DELETED;
        int nOrg = ld1(M.tn, pOppTri, m3(pOppOri + 1)), nApex = ld1(M.tn, index, m3(ori + 2));
        int npDest = ld1(M.tn, t2, m3(t2_ori + 1)), npApex = ld1(M.tn, t1, m3(t1_ori + 2));
        set_tri(M, pOrg, pO, pApex, index, ori);
        set_tri(M, pApex, pO, nOpp, t1, t1_ori);
        set_link(sl, nOrg + 3, kMaxInt, nApex + 3, 4 * pos, ori);
        set_link(sl, kMaxInt, npDest + 3, npApex + 3, 4 * pos + 2, t1_ori);
        sl[(4 * pos + 1) * 3 + m3(pOppOri + 1)] = nOrg + 3;
        sl[(4 * pos + 3) * 3 + m3(t2_ori + 1)] = npDest + 3;
        sOrg = ld1(M.tsg, pOppTri, m3(pOppOri + 1));
        sDest = ld1(M.tsg, index, m3(ori + 1));
        sApex = ld1(M.tsg, index, m3(ori + 2));
        snOrg = ld1(M.tsg, t1, t1_ori);
        snDest = ld1(M.tsg, t2, m3(t2_ori + 1));
        snApex = ld1(M.tsg, t1, m3(t1_ori + 2));
      }
      int4 a, b;
      setc(a, ori, sOrg);
      setc(a, m3(ori + 1), sDest);
      setc(a, m3(ori + 2), sApex);
      a.w = 0;
      setc(b, t1_ori, snOrg);
      setc(b, m3(t1_ori + 1), snDest);
      setc(b, m3(t1_ori + 2), snApex);
      b.w = 0;
      M.tsg[index] = a;
      M.tsg[t1] = b;
      if (sOrg != -1) ps.add(sOrg, (index << 2) | ori, 7);
      if (sDest != -1) ps.add(sDest, (index << 2) | m3(ori + 1), 8);
      if (sApex != -1) ps.add(sApex, (index << 2) | m3(ori + 2), 9);
      if (snOrg != -1) ps.add(snOrg, (t1 << 2) | t1_ori, 10);
      if (snDest != -1) ps.add(snDest, (t1 << 2) | m3(t1_ori + 1), 11);
      if (snApex != -1) ps.add(snApex, (t1 << 2) | m3(t1_ori + 2), 12);
      M.tst[index] |= TS_CHECK;
      M.tst[t1] |= TS_CHECK;
      M.tst[pOppTri] &= (uint8_t)~TS_NOTNULL;
      M.tst[t2] &= (uint8_t)~TS_NOTNULL;
    }
  }
}

// updateNeighborlink (refine.cu:1554-1596) through tpos
__device__ __forceinline__ void p2_link(const Mesh &M, const int *ll, int *sl, int nlist, int nlink, int neighbor) {
  int tempIndex = dtri(nlink);
  if (tempIndex == -1) return;
  int w = M.tmark[tempIndex];
  if (w == kMaxInt || w < 0 || M.tfo[w] == 15) return;
  int li = M.tpos[tempIndex];
  if (li < 0 || li >= nlist || ll[li] != tempIndex || ll[li & ~3] != w) return;
  sl[li * 3 + dori(nlink)] = -neighbor;
}

// kernelUpdatePhase2, refine.cu:1598-1871
GQM_KERNEL void k_phase2(Mesh M, const int *win, const int *dn, const int *ll, int *sl) {
  int n = *dn;
  int nlist = 4 * n;
  GS_LOOP(pos, n) {
    int index = win[pos];
    int ori = M.tfo[index];
    if (ori < 3) {
      int pOpp = ld1(M.tn, index, m3(ori + 1));
      int pOppTri = dtri(pOpp), pOppOri = dori(pOpp);
      int4 ni = M.tn[index], np = M.tn[pOppTri];
      p2_link(M, ll, sl, nlist, comp(ni, ori), etri(index, ori));
      p2_link(M, ll, sl, nlist, comp(ni, m3(ori + 2)), etri(pOppTri, pOppOri));
      p2_link(M, ll, sl, nlist, comp(np, m3(pOppOri + 1)), etri(index, m3(ori + 1)));
      p2_link(M, ll, sl, nlist, comp(np, m3(pOppOri + 2)), etri(pOppTri, m3(pOppOri + 2)));
    } else if (ori < 6) {
      ori = m3(ori - 3 + 1);
      int t1 = ld1(M.tn, index, ori), t2 = ld1(M.tn, index, m3(ori + 2));
      int t1_ori = dori(t1), t2_ori = dori(t2);
      t1 = dtri(t1);
      t2 = dtri(t2);
      p2_link(M, ll, sl, nlist, ld1(M.tn, t1, m3(t1_ori + 2)), etri(index, ori));
      p2_link(M, ll, sl, nlist, ld1(M.tn, index, m3(ori + 1)), etri(index, m3(ori + 1)));
      p2_link(M, ll, sl, nlist, ld1(M.tn, t2, m3(t2_ori + 1)), etri(index, m3(ori + 2)));
    } else {
      ori -= 6;
      int pOpp = ld1(M.tn, index, ori);
      int pOppTri = dtri(pOpp), pOppOri = dori(pOpp);
      if (flip42_outward(M, pOppTri, pOppOri)) {
        int t1 = ld1(M.tn, index, m3(ori + 2)), t2 = ld1(M.tn, pOppTri, m3(pOppOri + 1));
        int t1_ori = dori(t1), t2_ori = dori(t2);
        t1 = dtri(t1);
        t2 = dtri(t2);
        p2_link(M, ll, sl, nlist, ld1(M.tn, pOppTri, m3(pOppOri + 2)), etri(index, ori));
        p2_link(M, ll, sl, nlist, ld1(M.tn, index, m3(ori + 1)), etri(index, m3(ori + 1)));
        p2_link(M, ll, sl, nlist, ld1(M.tn, t1, m3(t1_ori + 1)), etri(t1, m3(t1_ori + 1)));
        p2_link(M, ll, sl, nlist, ld1(M.tn, t2, m3(t2_ori + 2)), etri(t1, m3(t1_ori + 2)));
      } else {
        int t1 = ld1(M.tn, index, m3(ori + 1)), t2 = ld1(M.tn, pOppTri, m3(pOppOri + 2));
        int t1_ori = dori(t1), t2_ori = dori(t2);
        t1 = dtri(t1);
        t2 = dtri(t2);
        p2_link(M, ll, sl, nlist, ld1(M.tn, pOppTri, m3(pOppOri + 1)), etri(index, ori));
        p2_link(M, ll, sl, nlist, ld1(M.tn, index, m3(ori + 2)), etri(index, m3(ori + 2)));
        p2_link(M, ll, sl, nlist, ld1(M.tn, t2, m3(t2_ori + 1)), etri(t1, m3(t1_ori + 1)));
        p2_link(M, ll, sl, nlist, ld1(M.tn, t1, m3(t1_ori + 2)), etri(t1, m3(t1_ori + 2)));
      }
    }
  }
}

// resetEncseg, refine.cu:1879-1922
__device__ void reset_encseg(const Mesh &M, int s, int otri0, int otri1) {
  int e = -1;
  if (otri0 != -1) {
    int t = dtri(otri0), o = dori(otri0);
    int4 v = M.tv[t];
    if (encroached(M.pts[comp(v, m3(o + 1))], M.pts[comp(v, m3(o + 2))], M.pts[comp(v, o)], M.gc2, M.mode)) e = 0;
  }
  if (otri1 != -1) {
    int t = dtri(otri1), o = dori(otri1);
    int4 v = M.tv[t];
    if (encroached(M.pts[comp(v, m3(o + 1))], M.pts[comp(v, m3(o + 2))], M.pts[comp(v, o)], M.gc2, M.mode)) e = 0;
  }
  M.enc[s] = e;
}
// A link slot still holding "original neighbour + 3" means that neighbour is
// not part of a winning flip: point it back at us (refine.cu:1974-1992).
__device__ __forceinline__ int unlink_slot(const Mesh &M, int v, int newlink) {
  if (v > 0) {
    v = -(v - 3);
    int t = -v;
    if (t >= 0) st1(M.tn, dtri(t), dori(t), newlink);
  }
  return v;
}

// kernelUpdatePhase3, refine.cu:1924-2296
template <class SetFlag>
__device__ void phase3_body(const Mesh &M, int pos, int index, const int *sl, const SetFlag &set_flag) {
  {
    int ori = M.tfo[index];
    M.tfo[index] = 15;
    if (ori < 3) {
      int pOpp = ld1(M.tn, index, m3(ori + 1));
      int pOppTri = dtri(pOpp), pOppOri = dori(pOpp);
      int nOrg = sl[4 * pos * 3 + ori], nApex = sl[4 * pos * 3 + m3(ori + 2)];
      int npDest = sl[(4 * pos + 1) * 3 + m3(pOppOri + 1)], npApex = sl[(4 * pos + 1) * 3 + m3(pOppOri + 2)];
      nOrg = unlink_slot(M, nOrg, etri(index, ori));
      nApex = unlink_slot(M, nApex, etri(pOppTri, pOppOri));
      npDest = unlink_slot(M, npDest, etri(index, m3(ori + 1)));
      npApex = unlink_slot(M, npApex, etri(pOppTri, m3(pOppOri + 2)));
      int4 a, b;
      setc(a, ori, -nOrg);
      setc(a, m3(ori + 1), -npDest);
      setc(a, m3(ori + 2), etri(pOppTri, m3(pOppOri + 1)));
      a.w = 0;
      setc(b, pOppOri, -nApex);
      setc(b, m3(pOppOri + 1), etri(index, m3(ori + 2)));
      setc(b, m3(pOppOri + 2), -npApex);
      b.w = 0;
      M.tn[index] = a;
      M.tn[pOppTri] = b;
      int sOrg = ld1(M.tsg, index, ori), sDest = ld1(M.tsg, index, m3(ori + 1));
      int spOrg = ld1(M.tsg, pOppTri, pOppOri), spApex = ld1(M.tsg, pOppTri, m3(pOppOri + 2));
      if (sOrg != -1) reset_encseg(M, sOrg, (index << 2) | ori, -nOrg);
      if (sDest != -1) reset_encseg(M, sDest, (index << 2) | m3(ori + 1), -npDest);
      if (spOrg != -1) reset_encseg(M, spOrg, (pOppTri << 2) | pOppOri, -nApex);
      if (spApex != -1) reset_encseg(M, spApex, (pOppTri << 2) | m3(pOppOri + 2), -npApex);
      set_flag(pOppTri);
    } else if (ori < 6) {
      ori = m3(ori - 3 + 1);
      int t1 = ld1(M.tn, index, ori), t2 = ld1(M.tn, index, m3(ori + 2));
      int t1_ori = dori(t1), t2_ori = dori(t2);
      t1 = dtri(t1);
      t2 = dtri(t2);
      int nOrg = sl[(4 * pos + 1) * 3 + m3(t1_ori + 2)], nDest = sl[4 * pos * 3 + m3(ori + 1)];
      int nApex = sl[(4 * pos + 2) * 3 + m3(t2_ori + 1)];
      nOrg = unlink_slot(M, nOrg, etri(index, ori));
      nDest = unlink_slot(M, nDest, etri(index, m3(ori + 1)));
      nApex = unlink_slot(M, nApex, etri(index, m3(ori + 2)));
      int4 a;
      setc(a, ori, -nOrg);
      setc(a, m3(ori + 1), -nDest);
      setc(a, m3(ori + 2), -nApex);
      a.w = 0;
      M.tn[index] = a;
      int4 s = M.tsg[index];
      int sOrg = comp(s, ori), sDest = comp(s, m3(ori + 1)), sApex = comp(s, m3(ori + 2));
      if (sOrg != -1) reset_encseg(M, sOrg, (index << 2) | ori, -nOrg);
      if (sDest != -1) reset_encseg(M, sDest, (index << 2) | m3(ori + 1), -nDest);
      if (sApex != -1) reset_encseg(M, sApex, (index << 2) | m3(ori + 2), -nApex);
      M.tflip[t1] = 0;
      M.tflip[t2] = 0;
    } else {
      ori -= 6;
      int pOpp = ld1(M.tn, index, ori);
      int pOppTri = dtri(pOpp), pOppOri = dori(pOpp);
      bool outward = flip42_outward(M, pOppTri, pOppOri);
      int t1, t2, t1_ori, t2_ori;
      if (outward) {
        t1 = ld1(M.tn, index, m3(ori + 2));
        t2 = ld1(M.tn, pOppTri, m3(pOppOri + 1));
        t1_ori = dori(t1);
        t2_ori = dori(t2);
        t1 = dtri(t1);
        t2 = dtri(t2);
        int nOrg = sl[(4 * pos + 1) * 3 + m3(pOppOri + 2)], nDest = sl[4 * pos * 3 + m3(ori + 1)];
        int npDest = sl[(4 * pos + 2) * 3 + m3(t1_ori + 1)], npApex = sl[(4 * pos + 3) * 3 + m3(t2_ori + 2)];
        nOrg = unlink_slot(M, nOrg, etri(index, ori));
        nDest = unlink_slot(M, nDest, etri(index, m3(ori + 1)));
        npDest = unlink_slot(M, npDest, etri(t1, m3(t1_ori + 1)));
        npApex = unlink_slot(M, npApex, etri(t1, m3(t1_ori + 2)));
        st1(M.tn, index, ori, -nOrg);
        st1(M.tn, index, m3(ori + 1), -nDest);
        st1(M.tn, t1, m3(t1_ori + 1), -npDest);
        st1(M.tn, t1, m3(t1_ori + 2), -npApex);
        int sOrg = ld1(M.tsg, index, ori), sDest = ld1(M.tsg, index, m3(ori + 1));
        int spDest = ld1(M.tsg, t1, m3(t1_ori + 1)), spApex = ld1(M.tsg, t1, m3(t1_ori + 2));
        if (sOrg != -1) reset_encseg(M, sOrg, (index << 2) | ori, -nOrg);
        if (sDest != -1) reset_encseg(M, sDest, (index << 2) | m3(ori + 1), -nDest);
        if (spDest != -1) reset_encseg(M, spDest, (t1 << 2) | m3(t1_ori + 1), -npDest);
        if (spApex != -1) reset_encseg(M, spApex, (t1 << 2) | m3(t1_ori + 2), -npApex);
      } else {
        t1 = ld1(M.tn, index, m3(ori + 1));
        t2 = ld1(M.tn, pOppTri, m3(pOppOri + 2));
        t1_ori = dori(t1);
        t2_ori = dori(t2);
        t1 = dtri(t1);
        t2 = dtri(t2);
        int nOrg = sl[(4 * pos + 1) * 3 + m3(pOppOri + 1)], nApex = sl[4 * pos * 3 + m3(ori + 2)];
        int npDest = sl[(4 * pos + 3) * 3 + m3(t2_ori + 1)], npApex = sl[(4 * pos + 2) * 3 + m3(t1_ori + 2)];
        nOrg = unlink_slot(M, nOrg, etri(index, ori));
        nApex = unlink_slot(M, nApex, etri(index, m3(ori + 2)));
        npDest = unlink_slot(M, npDest, etri(t1, m3(t1_ori + 1)));
        npApex = unlink_slot(M, npApex, etri(t1, m3(t1_ori + 2)));
        st1(M.tn, index, ori, -nOrg);
        st1(M.tn, index, m3(ori + 2), -nApex);
        st1(M.tn, t1, m3(t1_ori + 1), -npDest);
        st1(M.tn, t1, m3(t1_ori + 2), -npApex);
        int sOrg = ld1(M.tsg, index, ori), sApex = ld1(M.tsg, index, m3(ori + 2));
        int spDest = ld1(M.tsg, t1, m3(t1_ori + 1)), spApex = ld1(M.tsg, t1, m3(t1_ori + 2));
        if (sOrg != -1) reset_encseg(M, sOrg, (index << 2) | ori, -nOrg);
        if (sApex != -1) reset_encseg(M, sApex, (index << 2) | m3(ori + 2), -nApex);
        if (spDest != -1) reset_encseg(M, spDest, (t1 << 2) | m3(t1_ori + 1), -npDest);
        if (spApex != -1) reset_encseg(M, spApex, (t1 << 2) | m3(t1_ori + 2), -npApex);
      }
      set_flag(t1);
      M.tflip[pOppTri] = 0;
      M.tflip[t2] = 0;
    }
  }
}


// kernelMarkReduantPoints, refine.cu:604-677
GQM_KERNEL void k_mark_redundant(Mesh M, int *delmarker, const int *dellist, const int *dn) {
  int n = *dn;
  GS_LOOP(pos, n) {
    int out = -1;
    int sindex = dellist[pos];
    int otri = s2t_get(M, sindex);
    int t = dtri(otri), o = dori(otri);
    int4 v = M.tv[t];
    int pApex = comp(v, o);
    double2 vO = M.pts[comp(v, m3(o + 1))], vD = M.pts[comp(v, m3(o + 2))], vA = M.pts[pApex];
    uint8_t s = M.ps[pApex];
    if ((s & PS_STEINER) && !(s & PS_SEGSPLIT) &&
        ((vO.x - vA.x) * (vD.x - vA.x) + (vO.y - vA.y) * (vD.y - vA.y) < 0.0)) {
      M.pred[pApex] = 1;
      mark_fan(M, t, m3(o + 2));
      out = sindex;
    }
    int on = ld1(M.tn, t, o);
    if (on != -1) {
      t = dtri(on);
      o = dori(on);
      pApex = ld1(M.tv, t, o);
      vA = M.pts[pApex];
      s = M.ps[pApex];
      if ((s & PS_STEINER) && !(s & PS_SEGSPLIT) &&
          ((vO.x - vA.x) * (vD.x - vA.x) + (vO.y - vA.y) * (vD.y - vA.y) < 0.0)) {
        M.pred[pApex] = 1;
        mark_fan(M, t, m3(o + 2));
        out = sindex;
      }
    }
    delmarker[pos] = out;
  }
}

// ============================================================================
// Flip-flop driven by active sets.  The reference rescans every triangle slot
// several times per flip step (refine.cu:2356-2489).  Here a step works on
//   A : the triangles whose flip flag is set (built from queue Q),
//   T : the triangles claimed in the step (tmark reset at the next step),
//   W : the winners,
// and every flag set during a step pushes its triangle onto the next queue,
// deduplicated by a generation stamp.  The per-triangle results are the
// reference's: no kernel below depends on the order of its list.
// ============================================================================
// Control block of a flip-flop loop, resident on the device so that the loop
// can run as a CUDA graph with a device-side condition.
// Launch timer of one kernel inside the device-side flip loop, where CUDA
// events cannot bracket single launches.  Each block stamps %globaltimer when
// it starts and when it ends; the last block to finish adds (latest end -
// earliest start) to the total, i.e. the launch's execution time from its
// first block to its last, and counts the launch and its items.
struct KTimer {
  unsigned long long t0, t1;  // earliest block start / latest block end of the current launch
  unsigned long long total_ns, launches, items;
  unsigned long long winners;  // flips and flops applied (small-step kernel)
  unsigned long long first_items[4];  // items of the first four launches since the reset
  unsigned blocks_done;
  int on;
};
__device__ __forceinline__ unsigned long long global_ns() {
#ifdef GQM_HOST_EMU
  return (unsigned long long)std::chrono::duration_cast<std::chrono::nanoseconds>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
#else
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
#endif
}
// called by every thread of the block after its work, with the block's start
// stamp; the last block's `items` and `winners` are added for the launch
__device__ __forceinline__ void ktimer_end(KTimer *tm, unsigned long long start, long long items,
                                           long long winners = 0) {
  __syncthreads();
  if (threadIdx.x == 0) {
    atomicMin(&tm->t0, start);
    atomicMax(&tm->t1, global_ns());
    __threadfence();
    unsigned done = atomicAdd(&tm->blocks_done, 1u);
    if (done == gridDim.x - 1) {
      __threadfence();
      volatile KTimer *v = tm;
      v->total_ns += v->t1 - v->t0;
      if (v->launches < 4) v->first_items[v->launches] = (unsigned long long)items;
      v->launches += 1;
      v->items += (unsigned long long)items;
      v->winners += (unsigned long long)winners;
      v->t0 = ~0ull;
      v->t1 = 0;
      v->blocks_done = 0;
    }
  }
}
GQM_KERNEL void k_ktimer_reset(KTimer *tm, int on) {
  if (GQM_BLOCK0 && threadIdx.x == 0) {
    tm->t0 = ~0ull;
    tm->t1 = 0;
    tm->total_ns = tm->launches = tm->items = tm->winners = 0;
    for (int i = 0; i < 4; ++i) tm->first_items[i] = 0;
    tm->blocks_done = 0;
    tm->on = on;
  }
}

constexpr int kFlipProfileBins = 32;
struct FlipCtl {
  int gen;          // generation of the stamps of the current step
  unsigned epoch;   // launch epoch of the subseg2tri stores (all kernels share it)
  int nact;         // |A|
  int nact_next;    // |A| of the next step, counted by k_flip_reset_filter
  int winn;         // |W|
  int qn;           // length of the next queue
  int tn;           // number of claimed triangles
  int steps;        // flip steps executed (all loops)
  int small_steps;  // of which steps run by the single-block kernel (k_flip_small)
  int entry_steps;  // steps at entry of the current loop
  int cap_hit;      // the step bound stopped a loop
  int cond;         // loop condition of the last step
  long long cap;    // bound on the steps of one loop
  int *errp;        // device error word (GQM_ERR_ROUND_LIMIT on cap_hit)
  // device time of the loops (%globaltimer at loop entry, summed at loop end)
  unsigned long long loop_t0, loop_ns, loops;
  // step profile of the run: steps and active triangles by floor(log2 |A|)
  unsigned long long prof_steps[kFlipProfileBins], prof_items[kFlipProfileBins];
};
struct FlipQ {
  int *q;           // next queue
  int *qn;          // its length
  const int *genp;  // generation of the next queue
};
__device__ __forceinline__ void push_flag(const Mesh &M, const FlipQ &Q, int t) {
  M.tflip[t] = 1;
  int g = *Q.genp;
  if (atomicExch(M.fstamp + t, g) != g) Q.q[list_slot(Q.qn)] = t;
}
struct TouchL {
  int *l;
  int *n;
  const int *genp;
};
__device__ __forceinline__ void touch(const Mesh &M, const TouchL &T, int t) {
  int g = *T.genp;
  if (atomicExch(M.tstamp + t, g) != g) T.l[list_slot(T.n)] = t;
}
__device__ __forceinline__ void claim(const Mesh &M, const TouchL &T, int t, int v) {
  atomicMin(M.tmark + t, v);
  touch(M, T, t);
}

// Loop condition of a flip-flop step (refine.cu:2489: continue while any
// triangle is flagged), with a bound on the steps of one loop.  On continue,
// the counters of the next step are prepared here.
__device__ __forceinline__ int flip_next(FlipCtl *c) {
  int cond = c->nact > 0;
  if (cond) {
    int b = 31 - __clz(c->nact);
    c->prof_steps[b]++;
    c->prof_items[b] += (unsigned long long)c->nact;
  }
  if (cond && (long long)(c->steps - c->entry_steps) >= c->cap) {
    cond = 0;
    c->cap_hit = 1;
    atomicCAS(c->errp, 0, -2);
  }
  if (cond) {
    c->gen++;
    c->epoch++;
    c->winn = 0;
    c->qn = 0;
    c->tn = 0;
    c->steps++;
  } else {
    c->loop_ns += global_ns() - c->loop_t0;
    c->loops++;
  }
  c->cond = cond;
  return cond;
}
GQM_KERNEL void k_flip_prep(FlipCtl *c, cudaGraphConditionalHandle h, int use_graph) {
  if (GQM_BLOCK0 && threadIdx.x == 0) {
    c->entry_steps = c->steps;
    c->nact_next = 0;
    c->loop_t0 = global_ns();
    int cond = flip_next(c);
#ifndef GQM_HOST_EMU
    if (use_graph) cudaGraphSetConditional(h, cond);
#endif
    (void)cond;
    (void)use_graph;
    (void)h;
  }
}
GQM_KERNEL void k_flip_cond(FlipCtl *c, cudaGraphConditionalHandle h, int use_graph) {
  if (GQM_BLOCK0 && threadIdx.x == 0) {
    c->nact = c->nact_next;  // the filtered queue of this step is the next step's A
    c->nact_next = 0;
    int cond = flip_next(c);
#ifndef GQM_HOST_EMU
    if (use_graph) cudaGraphSetConditional(h, cond);
#endif
    (void)cond;
    (void)use_graph;
    (void)h;
  }
}
GQM_KERNEL void k_bump_epoch(FlipCtl *c) {
  if (GQM_BLOCK0 && threadIdx.x == 0) c->epoch++;
}
// per-run reset of the control block; gen and epoch keep growing across runs
// so that stamps and subseg2tri tags left by earlier runs never collide
GQM_KERNEL void k_ctl_reset(FlipCtl *c, long long cap, int *errp) {
  if (GQM_BLOCK0 && threadIdx.x < kFlipProfileBins) {
    c->prof_steps[threadIdx.x] = 0;
    c->prof_items[threadIdx.x] = 0;
  }
  if (GQM_BLOCK0 && threadIdx.x == 0) {
    c->steps = 0;
    c->small_steps = 0;
    c->entry_steps = 0;
    c->cap_hit = 0;
    c->cond = 0;
    c->cap = cap;
    c->errp = errp;
  }
}


// reset tmark / tfo before the first step of a flip-flop
template <class N>
GQM_KERNEL void k_flip_entry_reset(Mesh M, N ntri_) {
  const int ntri = nval(ntri_);
  GS_LOOP(t, ntri) {
    M.tmark[t] = kMaxInt;
    M.tfo[t] = 15;
  }
}
// A = queue entries whose flag is still set on a live triangle
GQM_KERNEL void k_flip_filter(Mesh M, const int *q, const int *qn, int *act, int *actn) {
  int n = *qn;
  GS_LOOP(k, n) {
    int t = q[k];
    if (M.tflip[t] && (M.tst[t] & TS_NOTNULL)) act[list_slot(actn)] = t;
  }
}
// tmark of the triangles claimed in this step back to "unclaimed"; also
// empties A for the filter that follows (A is not read after the winners).
GQM_KERNEL void k_flip_reset_touched(Mesh M, const int *tl, const int *tn, int *nact) {
  int n = *tn;
  GS_LOOP(k, n) M.tmark[tl[k]] = kMaxInt;
  if (GQM_BLOCK0 && threadIdx.x == 0) *nact = 0;
}
// k_flip_reset_touched and k_flip_filter in one launch: the claims of this
// step are cleared and the next A is built (counted in *nextn, which
// k_flip_cond moves to |A|); the two loops touch disjoint fields.
GQM_KERNEL void k_flip_reset_filter(Mesh M, const int *tl, const int *tn, const int *q, const int *qn, int *act,
                                    int *nextn) {
  const int nt = *tn, nq = *qn;
  GS_LOOP(k, nt) M.tmark[tl[k]] = kMaxInt;
  GS_LOOP(k, nq) {
    const int t = q[k];
    if (M.tflip[t] && (M.tst[t] & TS_NOTNULL)) act[list_slot(nextn)] = t;
  }
}

// kernelCheckFlipping (refine.cu:778-1070) on A.  No flag is cleared here
// (the decision is kept in clr[k] and applied by k_flip_winner2), so the
// neighbour flags read below are the ones the step started with.  MINB is the
// grid-mode register budget: at least MINB resident 256-thread blocks per SM
// (2: at most 128 registers, some spilled; 1: up to 255, none spilled).
template <int PRED, int MINB = GQM_WALK_MIN_BLOCKS>
GQM_KERNEL void GQM_BOUNDS(MINB) k_check_flip2(Mesh M, const int *act, const int *dn, uint8_t *clr, TouchL T,
                                               KTimer *tm) {
  const int timed = tm->on;
  const unsigned long long start = timed ? global_ns() : 0;
  int n = *dn;
  GS_LOOP(k, n) {
    int index = act[k];
    int4 p = M.tv[index];
    int4 nb = M.tn[index];
    int4 sg = M.tsg[index];
    int pp[3] = {p.x, p.y, p.z};
    const bool red[3] = {is_red(M, p.x), is_red(M, p.y), is_red(M, p.z)};
    double2 v[3] = {M.pts[p.x], M.pts[p.y], M.pts[p.z]};
    // The gathers of all three edges are issued before any decision below:
    // nothing they read changes during the launch (flags are the ones the
    // step started with), so the edges are still decided in the reference's
    // order, but an item waits for two dependent levels of loads instead of
    // two per edge in turn.
    int eTri[3], eOri[3], eOpp[3];
    uint8_t eFlip[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const int tri = comp(nb, i);
      eTri[i] = dtri(tri);
      eOri[i] = dori(tri);
      const bool use = comp(sg, i) == -1 && eTri[i] >= 0;
      eFlip[i] = (use && eTri[i] < index) ? M.tflip[eTri[i]] : 0;
      eOpp[i] = use ? ld1(M.tv, eTri[i], eOri[i]) : -1;
    }
    bool eRed[3];
    double2 eV[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      eRed[i] = eOpp[i] >= 0 && is_red(M, eOpp[i]);
      eV[i] = eOpp[i] >= 0 ? M.pts[eOpp[i]] : v[i];
    }
    int mn = kMaxInt;
    for (int i = 0; i < 3; ++i)
      if (red[i] && pp[i] < mn) mn = pp[i];
    bool done = false;
#pragma unroll
    for (int i = 0; i < 3 && !done; i++) {
      if (mn == pp[i]) continue;
      if (comp(sg, i) != -1) continue;
      int pTri = eTri[i], pOri = eOri[i];
      if (!(index < pTri || (pTri >= 0 && !eFlip[i]))) continue;
      int pOpp = eOpp[i];
      if (eRed[i] && pOpp < mn) continue;
      double2 vOpp = eV[i];
      int org = m3(i + 1), dest = m3(i + 2), apex = i;
      if (mn != kMaxInt) {
        int deleteOri, n1, n2;
        if (mn == pp[org]) {
          deleteOri = m3(i + 2);
          n1 = comp(nb, dest);
          n2 = ld1(M.tn, pTri, m3(pOri + 1));
        } else {
          deleteOri = i;
          n1 = comp(nb, org);
          n2 = ld1(M.tn, pTri, m3(pOri + 2));
        }
        if (dtri(n1) == dtri(n2)) {  // 3-1 flip
          M.tfo[index] = (uint8_t)(3 + deleteOri);
          claim(M, T, index, index);
          claim(M, T, pTri, index);
          if (dtri(n1) >= 0) claim(M, T, dtri(n1), index);
          done = true;
          break;
        } else {
          int n1_tri = dtri(n1), n1_ori = dori(n1), n2_tri = dtri(n2), n2_ori = dori(n2);
          int n1_pOpp = ld1(M.tv, n1_tri, n1_ori), n2_pOpp = ld1(M.tv, n2_tri, n2_ori);
          double2 n1_vOpp = M.pts[n1_pOpp], n2_vOpp = M.pts[n2_pOpp];
          int n3 = (mn == pp[org]) ? ld1(M.tn, n1_tri, m3(n1_ori + 2)) : ld1(M.tn, n1_tri, m3(n1_ori + 1));
          if (dtri(n3) == dtri(n2)) {
            bool four = false;
            if (mn == pp[org]) {
              double d = orient<PRED>(v[apex], v[org], vOpp);
              if (d == 0) {
                double t0 = orient<PRED>(v[dest], v[apex], n1_vOpp);
                double t1 = orient<PRED>(v[dest], v[org], n1_vOpp);
                bool f0 = (t0 > 0 && t1 < 0);
                t0 = orient<PRED>(v[dest], v[org], n2_vOpp);
                t1 = orient<PRED>(v[dest], vOpp, n2_vOpp);
                bool f1 = (t0 > 0 && t1 < 0);
                four = (!f0 && !f1);
              }
            } else {
              double d = orient<PRED>(v[apex], v[dest], vOpp);
              if (d == 0) {
                double t0 = orient<PRED>(v[org], v[dest], n1_vOpp);
                double t1 = orient<PRED>(v[org], v[apex], n1_vOpp);
                bool f0 = (t0 > 0 && t1 < 0);
                t0 = orient<PRED>(v[org], vOpp, n2_vOpp);
                t1 = orient<PRED>(v[org], v[dest], n2_vOpp);
                bool f1 = (t0 > 0 && t1 < 0);
                four = (!f0 && !f1);
              }
            }
            if (four) {
              if (is_red(M, n1_pOpp) && n1_pOpp < mn) continue;
              M.tfo[index] = (uint8_t)(6 + i);
              claim(M, T, index, index);
              claim(M, T, pTri, index);
              claim(M, T, n1_tri, index);
              claim(M, T, n2_tri, index);
              done = true;
              break;
            }
          }
        }
        double t1 = orient<PRED>(v[apex], v[org], vOpp);
        if (t1 <= 0) continue;
        double t2 = orient<PRED>(v[apex], v[dest], vOpp);
        if (t2 >= 0) continue;
        M.tfo[index] = (uint8_t)m3(i + 2);
        claim(M, T, index, index);
        claim(M, T, pTri, index);
        done = true;
        break;
      }
      double ret = incircle<PRED>(v[apex], v[org], v[dest], vOpp);
      double ret_opp = incircle<PRED>(v[org], vOpp, v[dest], v[apex]);
      double ret_after = incircle<PRED>(v[apex], v[org], vOpp, v[dest]);
      double ret_after_opp = incircle<PRED>(vOpp, v[dest], v[apex], v[org]);
      if (ret > 0 && ret_opp > 0 && ret_after < 0 && ret_after_opp < 0) {
        int pa = pp[apex];
        uint8_t sa = M.ps[pa], so = M.ps[pOpp];
        int td = -1;
        if ((sa & PS_SEGSPLIT) && (so & PS_SEGSPLIT))
          td = -1;
        else if ((sa & PS_NEW) && (so & PS_NEW)) {
          if (sa & PS_SEGSPLIT)
            td = 1;
          else if (so & PS_SEGSPLIT)
            td = 0;
          else
            td = pa < pOpp ? 1 : 0;
        }
        if (td == -1) {
          M.tfo[index] = (uint8_t)m3(i + 2);
          claim(M, T, index, index);
          claim(M, T, pTri, index);
        } else if (td == 0) {
          claim(M, T, index, negate_idx(etri(index, m3(i + 2))));
        } else {
          int tv2 = negate_idx(etri(pTri, m3(pOri + 2)));
          claim(M, T, index, tv2);
          claim(M, T, pTri, tv2);
        }
        done = true;
        break;
      }
    }
    clr[k] = done ? 0 : 1;
  }
  if (timed) ktimer_end(tm, start, n);
}

// kernelMarkFlipWinner (refine.cu:1072-1170) on A; applies the deferred flag
// clears, re-queues the triangles that keep their flag, collects winners.
// Winner test of one entry of A (the body of kernelMarkFlipWinner); true when
// the triangle's flip won all the triangles it needs.
__device__ __forceinline__ bool flip_winner(const Mesh &M, const FlipQ &Q, int index, uint8_t clear) {
  if (clear) {
    M.tflip[index] = 0;
    return false;
  }
  push_flag(M, Q, index);
  int ori = M.tfo[index];
  if (ori == 15) return false;
  bool w = false;
  if (M.tmark[index] == index) {
    if (ori < 3) {
      int pOppTri = dtri(ld1(M.tn, index, m3(ori + 1)));
      w = (M.tmark[pOppTri] == index);
    } else if (ori < 6) {
      int o = m3(ori - 3 + 1);
      int t1 = dtri(ld1(M.tn, index, o)), t2 = dtri(ld1(M.tn, index, m3(o + 2)));
      w = (t1 < 0 || M.tmark[t1] == index) && (t2 < 0 || M.tmark[t2] == index);
    } else {
      int o = ori - 6;
      int pOpp = ld1(M.tn, index, o);
      int pOppTri = dtri(pOpp), pOppOri = dori(pOpp);
      int pOrg = ld1(M.tv, index, m3(o + 1)), pDest = ld1(M.tv, index, m3(o + 2));
      int t1, t2;
      if (is_red(M, pOrg) && (!is_red(M, pDest) || pOrg < pDest)) {
        t1 = ld1(M.tn, index, m3(o + 2));
        t2 = ld1(M.tn, pOppTri, m3(pOppOri + 1));
      } else {
        t1 = ld1(M.tn, index, m3(o + 1));
        t2 = ld1(M.tn, pOppTri, m3(pOppOri + 2));
      }
      t1 = dtri(t1);
      t2 = dtri(t2);
      w = (M.tmark[pOppTri] == index && M.tmark[t1] == index && M.tmark[t2] == index);
    }
  }
  if (!w) M.tfo[index] = 15;
  return w;
}
// The loop keeps whole warps together (the winner counts are added per warp).
GQM_KERNEL void k_flip_winner2(Mesh M, const int *act, const int *dn, const uint8_t *clr, FlipQ Q, int *win,
                               int *winn) {
  const int n = *dn;
  const int lane = (int)(threadIdx.x & 31u);
  for (int base = GQM_GTID - lane; base < n; base += GQM_GSIZE) {
    const int k = base + lane;
    const int index = k < n ? act[k] : -1;
    const bool w = k < n && flip_winner(M, Q, index, clr[k]);
    if (w) win[list_slot(winn)] = index;
    win_mark(M, index, w);
  }
}

// kernelInitLinklist + kernelUpdatePhase1 in one launch: each winner's list
// setup reads only triangles the winner owns, before its own phase-1 writes.
// The subseg2tri stores of phase 1 are made last, keyed by the winner's rank.
GQM_KERNEL void GQM_WALK_BOUNDS k_link_phase1(Mesh M, const int *win, const int *dn, int *ll, int *sl, const unsigned *ep) {
  const int n = *dn;
  const uint32_t epoch = *ep;
  GS_LOOP(pos, n) {
    const int index = win[pos];
    PendingS2T ps;
    ps.n = 0;
    init_link_body(M, pos, index, ll);
    phase1_body(M, pos, index, sl, ps);
    if (ps.n) {
      const int rank = win_rank(M, index);
      for (int i = 0; i < ps.n; ++i) s2t_store(M, ps.s[i], ps.v[i], epoch, wkey(rank, ps.slot[i]));
    }
  }
}

// kernelUpdatePhase3 (refine.cu:1924-2296) with flags pushed onto the queue
struct QueueFlag {
  const Mesh *M;
  const FlipQ *Q;
  __device__ void operator()(int t) const { push_flag(*M, *Q, t); }
};
GQM_KERNEL void k_phase3q(Mesh M, const int *win, const int *dn, const int *sl, FlipQ Q) {
  int n = *dn;
  QueueFlag f{&M, &Q};
  const int lane = (int)(threadIdx.x & 31u);
  for (int base = GQM_GTID - lane; base < n; base += GQM_GSIZE) {  // whole warps (see win_unmark)
    const int pos = base + lane;
    const int index = pos < n ? win[pos] : -1;
    if (pos < n) phase3_body(M, pos, index, sl, f);
    win_unmark(M, index, pos < n);  // phase 1 has read the bitmap
  }
}

// kernelMarkReduntantSteiner (refine.cu:2298-2326) over the claimed triangles
__device__ void mark_fan_q(const Mesh &M, const FlipQ &Q, int triIndex, int triOri) {
  int cur = triIndex, ori = triOri, guard = 0;
  do {
    push_flag(M, Q, cur);
    int nx = ld1(M.tn, cur, m3(ori + 2));
    cur = dtri(nx);
    ori = dori(nx);
    if (++guard > (1 << 20)) {
      raise_err(M, -4);
      return;
    }
  } while (cur > -1 && cur != triIndex);
}
GQM_KERNEL void k_mark_red_steiner_q(Mesh M, const int *tl, const int *dn, FlipQ Q) {
  int n = *dn;
  GS_LOOP(k, n) {
    int index = tl[k];
    if (M.tmark[index] >= 0) continue;
    int otri = negate_idx(M.tmark[index]);
    int triIndex = dtri(otri), triOri = dori(otri);
    if (triIndex != index) push_flag(M, Q, index);
    int p = ld1(M.tv, triIndex, m3(triOri + 1));
    M.pred[p] = 1;
    mark_fan_q(M, Q, triIndex, triOri);
  }
}

// ============================================================================
// Midpoint insertion (refine.cu:2492-3070)
// ============================================================================
__device__ __forceinline__ void reset_tri_and_nbrs(const Mesh &M, int t, bool mark) {
  if (mark) M.tmark[t] = kMaxInt;
  M.tfo[t] = 15;
  int4 nb = M.tn[t];
  if (nb.x != -1) M.tfo[dtri(nb.x)] = 15;
  if (nb.y != -1) M.tfo[dtri(nb.y)] = 15;
  if (nb.z != -1) M.tfo[dtri(nb.z)] = 15;
}
// kernelResetMidInsertionMarker, refine.cu:2492-2542
GQM_KERNEL void k_reset_mid(Mesh M, const int *mids, const int *dn, const int *imark) {
  int n = *dn;
  GS_LOOP(pos, n) {
    int sindex = imark[mids[pos]];
    int otri = s2t_get(M, sindex);
    int t = dtri(otri), o = dori(otri);
    reset_tri_and_nbrs(M, t, true);
    int on = ld1(M.tn, t, o);
    if (on != -1) reset_tri_and_nbrs(M, dtri(on), true);
  }
}
// kernelMarkMidInsertion, refine.cu:2544-2579
GQM_KERNEL void k_mark_mid(Mesh M, const int *mids, const int *dn, const int *imark) {
  int n = *dn;
  GS_LOOP(pos, n) {
    int sindex = imark[mids[pos]];
    int otri = s2t_get(M, sindex);
    int t = dtri(otri), o = dori(otri);
    atomicMin(M.tmark + t, sindex);
    int on = ld1(M.tn, t, o);
    if (on != -1) atomicMin(M.tmark + dtri(on), sindex);
  }
}
// Snapshot of subseg2tri for every candidate before any winner writes
// (the reference reads it at refine.cu:2636 in the same kernel that rewrites
// it at 2844-2850).
GQM_KERNEL void k_mid_snapshot(Mesh M, const int *mids, const int *dn, const int *imark, int *snap) {
  int n = *dn;
  GS_LOOP(pos, n) snap[pos] = s2t_get(M, imark[mids[pos]]);
}

// kernelInsertMidPoints, refine.cu:2594-2927 (debug printing left out)
template <class S, class N>
GQM_KERNEL void GQM_WALK_BOUNDS k_insert_mid(Mesh M, const int *mids, const int *dn, int *imark, const int *snap,
                                             S pslots_, S tslots_, N nsub_, const unsigned *ep,
                                             unsigned long long *counter) {
  const int *pslots = slots_of(pslots_), *tslots = slots_of(tslots_);
  const int nsub = nval(nsub_);
  int n = *dn;
  uint32_t epoch = *ep;
  GS_LOOP(pos, n) {
    int tindex = mids[pos];
    int sindex = imark[tindex];
    int otri = snap[pos];
    int tri[4], triOri[2];
    tri[0] = dtri(otri);
    triOri[0] = dori(otri);
    if (M.tmark[tri[0]] != sindex) continue;
    int4 s0 = M.tsg[tri[0]];
    bool acutedest = comp(s0, m3(triOri[0] + 1)) != -1;
    bool acuteorg = comp(s0, m3(triOri[0] + 2)) != -1;
    int4 n0 = M.tn[tri[0]];
    int on = comp(n0, triOri[0]);
    tri[2] = dtri(on);
    triOri[1] = dori(on);
    if (tri[2] != -1 && M.tmark[tri[2]] != sindex) continue;
    int4 s2 = make_int4(-1, -1, -1, 0);
    if (tri[2] != -1) {
      s2 = M.tsg[tri[2]];
      if (comp(s2, m3(triOri[1] + 1)) != -1) acuteorg = true;
      if (comp(s2, m3(triOri[1] + 2)) != -1) acutedest = true;
    }
    int newp = pslots[tindex];
    tri[1] = tslots[2 * tindex];
    tri[3] = tslots[2 * tindex + 1];
    M.ps[newp] = PS_STEINER | PS_NEW | PS_SEGSPLIT;
    M.pred[newp] = 0;
    M.enc[sindex] = -1;
    M.enc[nsub + tindex] = -1;
    int4 v0 = M.tv[tri[0]];
    int p[3] = {comp(v0, m3(triOri[0] + 1)), comp(v0, m3(triOri[0] + 2)), comp(v0, triOri[0])};
    double2 a = M.pts[p[0]], b = M.pts[p[1]], c = M.pts[p[2]];
    double segmentlength = sqrt(gqm_madd(a.x - b.x, a.x - b.x, (a.y - b.y) * (a.y - b.y)));
    double split = 0.5;
    if (acuteorg || acutedest) {
      double npt = 1.0;
      while (segmentlength > 3.0 * npt) npt *= 2.0;
      while (segmentlength < 1.5 * npt) npt *= 0.5;
      split = npt / segmentlength;
      if (acutedest) split = 1.0 - split;
    }
    double2 m = make_double2(gqm_madd(b.x - a.x, split, a.x), gqm_madd(b.y - a.y, split, a.y));
    double multiplier = gqm_orient_ref(a.x, a.y, b.x, b.y, m.x, m.y);
    double divisor = gqm_madd(a.x - b.x, a.x - b.x, (a.y - b.y) * (a.y - b.y));
    if ((multiplier != 0.0) && (divisor != 0.0)) {
      multiplier = multiplier / divisor;
      if (multiplier == multiplier) {
        m.x = gqm_madd(multiplier, b.y - a.y, m.x);
        m.y = gqm_madd(multiplier, a.x - b.x, m.y);
      }
    }
    M.pts[newp] = m;
    int seg[3] = {comp(s0, triOri[0]), comp(s0, m3(triOri[0] + 1)), comp(s0, m3(triOri[0] + 2))};
    M.tsg[tri[0]] = make_int4(seg[2], seg[0], -1, 0);
    M.tsg[tri[1]] = make_int4(seg[1], -1, nsub + tindex, 0);
    s2t_store(M, seg[0], (tri[0] << 2) | 1, epoch, wkey(pos, 0));
    s2t_store(M, nsub + tindex, (tri[1] << 2) | 2, epoch, wkey(pos, 1));
    M.s2seg[nsub + tindex] = M.s2seg[seg[0]];
    if (seg[1] != -1) s2t_store(M, seg[1], (tri[1] << 2) | 0, epoch, wkey(pos, 2));
    if (seg[2] != -1) s2t_store(M, seg[2], (tri[0] << 2) | 0, epoch, wkey(pos, 3));
    int e_s = -1, e_n = -1;
    if (encroached(a, m, c, M.gc2, M.mode)) e_s = 0;
    if (encroached(m, b, c, M.gc2, M.mode)) e_n = 0;
    int nb1 = comp(n0, m3(triOri[0] + 1)), nb2 = comp(n0, m3(triOri[0] + 2));
    M.tv[tri[0]] = make_int4(newp, p[2], p[0], 0);
    M.tv[tri[1]] = make_int4(newp, p[1], p[2], 0);
    if (tri[2] == -1) {
      M.tn[tri[0]] = make_int4(nb2, -1, (tri[1] << 2) | 1, 0);
      M.tn[tri[1]] = make_int4(nb1, (tri[0] << 2) | 2, -1, 0);
    } else {
      M.tn[tri[0]] = make_int4(nb2, (tri[2] << 2) | 2, (tri[1] << 2) | 1, 0);
      M.tn[tri[1]] = make_int4(nb1, (tri[0] << 2) | 2, (tri[3] << 2) | 1, 0);
    }
    M.tst[tri[0]] |= TS_CHECK;
    M.tflip[tri[0]] = 1;
    M.tfo[tri[0]] = 0;
    M.tst[tri[1]] = TS_NOTNULL | TS_CHECK;
    M.tflip[tri[1]] = 1;
    M.tfo[tri[1]] = 0;
    if (tri[2] != -1) {
      int sg2[3] = {comp(s2, triOri[1]), comp(s2, m3(triOri[1] + 1)), comp(s2, m3(triOri[1] + 2))};
      M.tsg[tri[2]] = make_int4(sg2[1], -1, sg2[0], 0);
      M.tsg[tri[3]] = make_int4(sg2[2], nsub + tindex, -1, 0);
      if (sg2[1] != -1) s2t_store(M, sg2[1], (tri[2] << 2) | 0, epoch, wkey(pos, 4));
      if (sg2[2] != -1) s2t_store(M, sg2[2], (tri[3] << 2) | 0, epoch, wkey(pos, 5));
      int4 v2 = M.tv[tri[2]];
      int q[3] = {comp(v2, m3(triOri[1] + 1)), comp(v2, m3(triOri[1] + 2)), comp(v2, triOri[1])};
      double2 qa = M.pts[q[0]], qb = M.pts[q[1]], qc = M.pts[q[2]];
      if (encroached(qa, m, qc, M.gc2, M.mode)) e_n = 0;
      if (encroached(m, qb, qc, M.gc2, M.mode)) e_s = 0;
      int4 n2 = M.tn[tri[2]];
      int m1 = comp(n2, m3(triOri[1] + 1)), m2 = comp(n2, m3(triOri[1] + 2));
      M.tv[tri[2]] = make_int4(newp, q[1], q[2], 0);
      M.tn[tri[2]] = make_int4(m1, (tri[3] << 2) | 2, (tri[0] << 2) | 1, 0);
      M.tv[tri[3]] = make_int4(newp, q[2], q[0], 0);
      M.tn[tri[3]] = make_int4(m2, (tri[1] << 2) | 2, (tri[2] << 2) | 1, 0);
      M.tst[tri[2]] |= TS_CHECK;
      M.tflip[tri[2]] = 1;
      M.tfo[tri[2]] = 0;
      M.tst[tri[3]] = TS_NOTNULL | TS_CHECK;
      M.tflip[tri[3]] = 1;
      M.tfo[tri[3]] = 0;
    }
    M.enc[sindex] = e_s;
    M.enc[nsub + tindex] = e_n;
    imark[tindex] = -1;
    count_event(counter);
  }
}

// Outer-edge relinking of new triangles (edge 0 faces outward), shared by
// kernelUpdateMidNeighbors (2929-3070) and kernelUpdateSteinerNeighbors
// (4902-5059).
__device__ void relink_outer(const Mesh &M, const int *tri, int iteration) {
  for (int i = 0; i < iteration; i++) {
    int curTri = tri[i];
    int seg = ld1(M.tsg, curTri, 0);
    int pOppTri = ld1(M.tn, curTri, 0);
    int pOpp = dtri(pOppTri), pOri = dori(pOppTri);
    int4 cv = M.tv[curTri];
    if (pOppTri < 0) {
      if (seg != -1) {
        M.enc[seg] = encroached(M.pts[cv.y], M.pts[cv.z], M.pts[cv.x], M.gc2, M.mode) ? 0 : -1;
      }
      continue;
    }
    if (M.tfo[pOpp] == 15) {
      st1(M.tn, pOpp, pOri, etri(curTri, 0));
      if (seg != -1) {
        double2 v0 = M.pts[cv.y], v1 = M.pts[cv.z], v2 = M.pts[cv.x];
        double2 v3 = M.pts[ld1(M.tv, pOpp, pOri)];
        bool e = encroached(v0, v1, v2, M.gc2, M.mode) || encroached(v1, v0, v3, M.gc2, M.mode);
        M.enc[seg] = e ? 0 : -1;
      }
    } else {
      for (int j = 0; j < 3; j++) {
        int neighbor = (j == 0) ? pOpp : dtri(ld1(M.tn, pOpp, j));
        if (neighbor > -1) {
          int4 nv = M.tv[neighbor];
          if (cv.y == nv.z && cv.z == nv.y) {
            st1(M.tn, neighbor, 0, etri(curTri, 0));
            if (seg != -1) {
              double2 v0 = M.pts[cv.y], v1 = M.pts[cv.z], v2 = M.pts[cv.x], v3 = M.pts[nv.x];
              bool e = encroached(v0, v1, v2, M.gc2, M.mode) || encroached(v1, v0, v3, M.gc2, M.mode);
              M.enc[seg] = e ? 0 : -1;
            }
            break;
          }
        }
      }
    }
  }
}

// kernelUpdateMidNeighbors, refine.cu:2929-3070
GQM_KERNEL void k_update_mid_nbrs(Mesh M, const int *mids, const int *dn, const int *imark, const int *enclist) {
  int n = *dn;
  GS_LOOP(pos, n) {
    int tindex = mids[pos];
    if (imark[tindex] != -1) continue;
    int sindex = enclist[tindex];
    int tri[4];
    tri[0] = dtri(s2t_get(M, sindex));
    int4 n0 = M.tn[tri[0]];
    tri[1] = dtri(n0.z);
    int iteration = (n0.y == -1) ? 2 : 4;
    tri[2] = dtri(n0.y);
    tri[3] = dtri(ld1(M.tn, tri[1], 2));
    relink_outer(M, tri, iteration);
  }
}

// kernelUpdatePStatus2Old, refine.cu:3072-3083
template <class N>
GQM_KERNEL void k_points_old(Mesh M, N npts_) {
  const int npts = nval(npts_);
  GS_LOOP(i, npts) {
    uint8_t s = M.ps[i];
    if (!(s & PS_DELETED)) M.ps[i] = (uint8_t)(s & ~PS_NEW);
  }
}

// ============================================================================
// Steiner points (refine.cu:3780-5105)
// ============================================================================
// computeCircumcenter, refine.cu:3780-3868
__device__ __forceinline__ double2 circumcenter(double2 vApex, double2 vOrg, double2 vDest, double offConstant,
                                                bool offcenter) {
  // gqm_madd: the products the reference's contracted build fuses (see
  // predicates.h); the sums are the same in either order
  double xdo = vDest.x - vOrg.x, ydo = vDest.y - vOrg.y;
  double xao = vApex.x - vOrg.x, yao = vApex.y - vOrg.y;
  double dodist = gqm_madd(xdo, xdo, ydo * ydo);
  double aodist = gqm_madd(xao, xao, yao * yao);
  double dadist = gqm_madd(vDest.x - vApex.x, vDest.x - vApex.x, (vDest.y - vApex.y) * (vDest.y - vApex.y));
  double tmp = xdo * yao - xao * ydo;
  double denominator = (tmp != 0) ? 0.5 / tmp : 0.5 / gqm_orient_ref(vDest.x, vDest.y, vApex.x, vApex.y, vOrg.x, vOrg.y);
  double dx = gqm_madd(yao, dodist, -(ydo * aodist)) * denominator;
  double dy = gqm_madd(xdo, aodist, -(xao * dodist)) * denominator;
  if (offcenter && (offConstant > 0.0)) {
    double dxoff, dyoff;
    if ((dodist < aodist) && (dodist < dadist)) {
      dxoff = 0.5 * xdo - offConstant * ydo;
      dyoff = gqm_madd(offConstant, xdo, 0.5 * ydo);
      if (gqm_madd(dxoff, dxoff, dyoff * dyoff) < gqm_madd(dx, dx, dy * dy)) {
        dx = dxoff;
        dy = dyoff;
      }
    } else if (aodist < dadist) {
      dxoff = 0.5 * xao + offConstant * yao;
      dyoff = 0.5 * yao - offConstant * xao;
      if (gqm_madd(dxoff, dxoff, dyoff * dyoff) < gqm_madd(dx, dx, dy * dy)) {
        dx = dxoff;
        dy = dyoff;
      }
    } else {
      dxoff = 0.5 * (vApex.x - vDest.x) - offConstant * (vApex.y - vDest.y);
      dyoff = gqm_madd(offConstant, vApex.x - vDest.x, 0.5 * (vApex.y - vDest.y));
      if (gqm_madd(dxoff, dxoff, dyoff * dyoff) < gqm_madd(dx - xdo, dx - xdo, (dy - ydo) * (dy - ydo))) {
        dx = xdo + dxoff;
        dy = ydo + dyoff;
      }
    }
  }
  return make_double2(vOrg.x + dx, vOrg.y + dy);
}

GQM_KERNEL void k_circumcenter(Mesh M, const int *bad, const int *dn, double offc, int offcenter, double2 *center) {
  int n = *dn;
  GS_LOOP(k, n) {
    int4 v = M.tv[bad[k]];
    center[k] = circumcenter(M.pts[v.x], M.pts[v.y], M.pts[v.z], offc, offcenter != 0);
  }
}

// kernelLocateSinkPoints, refine.cu:3908-4184
template <int PRED>
GQM_KERNEL void k_locate(Mesh M, const int *bad, const int *dn, const double2 *center, int *sinks) {
  int n = *dn;
  GS_LOOP(k, n) {
    int index = bad[k];
    if (!(M.tst[index] & TS_BAD)) {
      sinks[k] = -1;
      continue;
    }
    double2 cc = center[k];
    int curTri = index, curOri = 0;
    bool checkNeighbor = false, split = false;
    int dart = 3;
    int4 v = M.tv[curTri];
    double2 w0 = M.pts[v.x], w1 = M.pts[v.y], w2 = M.pts[v.z];
    double det0 = orient<PRED>(w0, w1, cc), det1 = orient<PRED>(w1, w2, cc), det2 = orient<PRED>(w2, w0, cc);
    int4 sg = M.tsg[index];
    if (det0 <= 0) {
      if (det0 == 0 || sg.z != -1) split = true;
      dart = 2;
    } else if (det1 <= 0) {
      if (det1 == 0 || sg.x != -1) split = true;
      dart = 0;
    } else if (det2 <= 0) {
      if (det2 == 0 || sg.y != -1) split = true;
      dart = 1;
    }
    if (!split && dart != 3) {
      int nb = ld1(M.tn, curTri, dart);
      if (nb < 0) {
        split = true;
      } else {
        curTri = dtri(nb);
        curOri = dori(nb);
        checkNeighbor = true;
      }
    }
    int guard = 0;
    while (checkNeighbor) {
      if (++guard > (1 << 24)) {
        raise_err(M, -3);
        break;
      }
      int4 tv = M.tv[curTri];
      double2 u[3] = {M.pts[tv.x], M.pts[tv.y], M.pts[tv.z]};
      dart = 3;
      int pOrg = m3(curOri + 1), pDest = m3(curOri + 2), pApex = curOri;
      double detLeft = orient<PRED>(u[pDest], u[pApex], cc);
      double detRight = orient<PRED>(u[pApex], u[pOrg], cc);
      bool moveleft;
      if (detLeft < 0.0) {
        if (detRight < 0.0)
          moveleft = gqm_madd(u[pDest].x - u[pOrg].x, cc.x - u[pApex].x,
                              (u[pDest].y - u[pOrg].y) * (cc.y - u[pApex].y)) >
                     0.0;
        else
          moveleft = true;
      } else {
        if (detRight < 0.0)
          moveleft = false;
        else {
          if (detLeft == 0.0) {
            split = true;
            dart = m3(curOri + 1);
            break;
          }
          if (detRight == 0.0) {
            split = true;
            dart = m3(curOri + 2);
            break;
          }
          break;
        }
      }
      dart = moveleft ? m3(curOri + 1) : m3(curOri + 2);
      int nb = ld1(M.tn, curTri, dart);
      if (nb < 0 || ld1(M.tsg, curTri, dart) != -1) {
        split = true;
        break;
      }
      curTri = dtri(nb);
      curOri = dori(nb);
    }
    atomicMin(M.tmark + curTri, index);
    if (split) {
      int nb = ld1(M.tn, curTri, dart);
      if (nb != -1) atomicMin(M.tmark + dtri(nb), index);
    }
    sinks[k] = (curTri << 2) | dart;
  }
}

// kernelRemoveLosers, refine.cu:4186-4235
GQM_KERNEL void k_remove_losers(Mesh M, const int *bad, const int *dn, const int *sinks, int *imark) {
  int n = *dn;
  GS_LOOP(k, n) {
    if (imark[k] < 0) continue;
    int sink = sinks[k] >> 2, dir = sinks[k] & 3, index = bad[k];
    if (M.tmark[sink] != index) {
      imark[k] = -1;
      continue;
    }
    if (dir != 3) {
      int nb = ld1(M.tn, sink, dir);
      if (nb != -1 && M.tmark[dtri(nb)] != index) imark[k] = -1;
    }
  }
}

// Cavity walk of kernelMarkCavities (4237-4368): depth-first over neighbours
// whose circumcircle contains the centre, not crossing subsegments except the
// sink's split edge, at most 50 triangles.  Returns the number of triangles in
// the cavity (stored, in visiting order, at out[j * stride]) or -1 when the
// cavity exceeds the cap.
//
// kernelCheckCavities (4422-4547) repeats the same walk and fails at the first
// triangle whose marker is not the candidate's.  Between the two launches only
// the markers change, never the mesh or the centres, so its walk visits exactly
// the triangles stored here (up to the first failure): checking the stored
// list gives the same verdict without a second walk or any predicate.
//
// The reference rescans a triangle's three edges from the first every time the
// walk comes back to it; the edges before the one it descended through were
// then rejected (circumcircle test false, a subsegment or the boundary) or lead
// to a triangle already in the region, and neither changes while the walk runs.
// So each stack frame keeps the edge to resume at: the same triangles are
// visited and claimed in the same order, each neighbour tested once.
//
// The three neighbours of a triangle are tested together when the walk first
// reaches it, with all their loads in flight at once (rows, then points), and
// the outcomes are kept in the frame; which edge the walk takes is still decided
// edge by edge from the resume point, with the region as it is then.  Nothing a
// test reads changes during the walk (only claim markers do), so the walk takes
// the same edges as one that tests each neighbour when it gets to it.
__device__ __forceinline__ unsigned cavity_hash(int t) { return ((unsigned)t * 2654435761u) >> 26; }
template <int PRED>
__device__ int cavity_walk(const Mesh &M, int sink, int direction, double2 cc, int badIndex, int *out,
                           int stride) {
  int region[kCavityCap], loop[kCavityCap];  // loop: (triangle << 2) | edge to resume at
  uint8_t inside[kCavityCap];                // per frame: neighbours whose circumcircle holds cc
  // one bit per hash of the region's triangles: a clear bit proves a triangle
  // is not in the region without scanning it (a set bit still scans)
  unsigned long long rbits = 0;
  int rsize = 0, lsize = 0;
  int cur = sink, start = 0;
  for (int guard = 0; guard < 4 * kCavityCap * 3 + 16; ++guard) {
    int4 nb = make_int4(-1, -1, -1, -1);
    if (start == 0) {  // first visit (a return always resumes past the edge it left by)
      if (rsize == kCavityCap || lsize == kCavityCap) return -1;
      region[rsize++] = cur;
      rbits |= 1ull << cavity_hash(cur);
      loop[lsize++] = cur << 2;
      atomicMin(M.tmark + cur, badIndex);
      const int4 sg = M.tsg[cur];
      nb = M.tn[cur];
      int tt[3];
      int4 q[3];
#pragma unroll
      for (int i = 0; i < 3; i++) {
        const int si = comp(sg, i);
        bool ok = comp(nb, i) != -1;
        if (cur == sink) {
          if (direction == 3 && si != -1) ok = false;
          if (direction < 3 && si != -1 && i != direction) ok = false;
        } else if (si != -1) {
          ok = false;
        }
        tt[i] = ok ? dtri(comp(nb, i)) : -1;
      }
#pragma unroll
      for (int i = 0; i < 3; i++)
        if (tt[i] >= 0) q[i] = M.tv[tt[i]];
      unsigned bits = 0;
#pragma unroll
      for (int i = 0; i < 3; i++)
        if (tt[i] >= 0 && incircle<PRED>(M.pts[q[i].x], M.pts[q[i].y], M.pts[q[i].z], cc) > 0) bits |= 1u << i;
      inside[lsize - 1] = (uint8_t)bits;
    } else if (inside[lsize - 1] >> start) {
      nb = M.tn[cur];
    }
    int nIdx = -1, taken = -1;
    const unsigned bits = inside[lsize - 1];
    for (int i = start; i < 3; i++) {
      if (!((bits >> i) & 1u)) continue;
      const int t = dtri(comp(nb, i));
      bool seen = false;
      if ((rbits >> cavity_hash(t)) & 1ull)
        for (int r = 0; r < rsize; ++r)
          if (region[r] == t) {
            seen = true;
            break;
          }
      if (seen) continue;
      nIdx = t;
      taken = i;
      break;
    }
    if (taken >= 0) {
      loop[lsize - 1] = (cur << 2) | (taken + 1);
      cur = nIdx;
      start = 0;
    } else {
      if (lsize > 0) lsize--;
      if (lsize == 0) {
        for (int j = 0; j < rsize; ++j) out[(long)j * stride] = region[j];
        return rsize;
      }
      cur = loop[lsize - 1] >> 2;
      start = loop[lsize - 1] & 3;
    }
  }
  raise_err(M, -6);
  return 0;
}

// kernelMarkCavities: claim every cavity triangle (atomicMin of the bad index);
// an oversized cavity makes its candidate an unconditional winner (negated
// index).  cavn[k] = stored cavity size (0 for an oversized one).
template <int PRED>
GQM_KERNEL void GQM_WALK_BOUNDS k_cavity_mark(Mesh M, const int *dn, const int *sinks, const double2 *center, const int *imark,
                              int *ilist, int *cav, int *cavn, int stride) {
  int n = *dn;
  GS_LOOP(k, n) {
    if (imark[k] < 0) continue;
    int badIndex = ilist[k];
    int c = cavity_walk<PRED>(M, sinks[k] >> 2, sinks[k] & 3, center[k], badIndex, cav + k, stride);
    if (c < 0) ilist[k] = negate_idx(badIndex);
    cavn[k] = c < 0 ? 0 : c;
  }
}
// kernelCheckCavities: a candidate loses if any triangle of its cavity was
// claimed by a smaller bad index.
GQM_KERNEL void k_cavity_check(Mesh M, const int *dn, const int *cav, const int *cavn, int stride, int *imark,
                               const int *ilist) {
  int n = *dn;
  GS_LOOP(k, n) {
    if (imark[k] < 0) continue;
    int badIndex = ilist[k];
    if (badIndex < 0) continue;
    int c = cavn[k];
    for (int j = 0; j < c; ++j)
      if (M.tmark[cav[(long)j * stride + k]] != badIndex) {
        imark[k] = -1;
        break;
      }
  }
}

// kernelMarkSteinerOnsegs, refine.cu:5061-5089
GQM_KERNEL void k_mark_onsegs(Mesh M, const int *wl, const int *dn, const int *sinks, int *encl2) {
  int n = *dn;
  GS_LOOP(w, n) {
    int sk = sinks[wl[w]];
    int index = sk >> 2, dir = sk & 3;
    if (dir != 3) {
      int sg = ld1(M.tsg, index, dir);
      if (sg != -1) encl2[sg] = 0;
    }
  }
}
// kernelResetSteinerInsertionMarker, refine.cu:4601-4649
GQM_KERNEL void k_reset_steiner(Mesh M, const int *wl, const int *dn, const int *sinks) {
  int n = *dn;
  GS_LOOP(w, n) {
    int sk = sinks[wl[w]];
    int index = sk >> 2, dir = sk & 3;
    reset_tri_and_nbrs(M, index, false);
    if (dir != 3) {
      int on = ld1(M.tn, index, dir);
      if (on != -1) reset_tri_and_nbrs(M, dtri(on), false);
    }
  }
}

// kernelInsertSteinerPoints, refine.cu:4651-4900
template <class S>
GQM_KERNEL void k_insert_steiner(Mesh M, const int *wl, const int *dn, const int *sinks, const double2 *center,
                                 S pslots_, S tslots_, const unsigned *ep, unsigned long long *counter) {
  const int *pslots = slots_of(pslots_), *tslots = slots_of(tslots_);
  int n = *dn;
  uint32_t epoch = *ep;
  GS_LOOP(pos, n) {
    int tindex = wl[pos];
    int index = sinks[tindex] >> 2, direction = sinks[tindex] & 3;
    int4 s0 = M.tsg[index];
    if (direction != 3 && comp(s0, direction) != -1) continue;
    int newp = pslots[pos];
    int nt1 = tslots[2 * pos], nt2 = tslots[2 * pos + 1];
    M.ps[newp] = PS_STEINER | PS_NEW;
    M.pred[newp] = 0;
    M.pts[newp] = center[tindex];
    int4 v0 = M.tv[index];
    int4 n0 = M.tn[index];
    if (direction == 3) {
      int t0 = index, t1 = nt1, t2 = nt2;
      M.tsg[t0] = make_int4(s0.x, -1, -1, 0);
      M.tsg[t1] = make_int4(s0.y, -1, -1, 0);
      M.tsg[t2] = make_int4(s0.z, -1, -1, 0);
      if (s0.x != -1) s2t_store(M, s0.x, (t0 << 2) | 0, epoch, wkey(pos, 0));
      if (s0.y != -1) s2t_store(M, s0.y, (t1 << 2) | 0, epoch, wkey(pos, 1));
      if (s0.z != -1) s2t_store(M, s0.z, (t2 << 2) | 0, epoch, wkey(pos, 2));
      // p[i] = vertex (i+1)%3 of the old triangle; neighbour[i] = old edge i
      M.tv[t0] = make_int4(newp, v0.y, v0.z, 0);
      M.tn[t0] = make_int4(n0.x, (t1 << 2) | 2, (t2 << 2) | 1, 0);
      M.tv[t1] = make_int4(newp, v0.z, v0.x, 0);
      M.tn[t1] = make_int4(n0.y, (t2 << 2) | 2, (t0 << 2) | 1, 0);
      M.tv[t2] = make_int4(newp, v0.x, v0.y, 0);
      M.tn[t2] = make_int4(n0.z, (t0 << 2) | 2, (t1 << 2) | 1, 0);
      M.tst[t0] |= TS_CHECK;
      M.tflip[t0] = 1;
      M.tfo[t0] = 0;
      M.tst[t1] = TS_NOTNULL | TS_CHECK;
      M.tflip[t1] = 1;
      M.tfo[t1] = 0;
      M.tst[t2] = TS_NOTNULL | TS_CHECK;
      M.tflip[t2] = 1;
      M.tfo[t2] = 0;
    } else {
      int o0 = direction;
      int otri = comp(n0, o0);
      int o1 = dori(otri);
      int tri0 = index, tri1 = nt1, tri2 = dtri(otri), tri3 = nt2;
      int p0 = comp(v0, m3(o0 + 1)), p1 = comp(v0, m3(o0 + 2)), p2 = comp(v0, o0);
      int seg[3] = {comp(s0, o0), comp(s0, m3(o0 + 1)), comp(s0, m3(o0 + 2))};
      M.tsg[tri0] = make_int4(seg[2], seg[0], -1, 0);
      M.tsg[tri1] = make_int4(seg[1], -1, seg[0], 0);
      if (seg[1] != -1) s2t_store(M, seg[1], (tri1 << 2) | 0, epoch, wkey(pos, 3));
      if (seg[2] != -1) s2t_store(M, seg[2], (tri0 << 2) | 0, epoch, wkey(pos, 4));
      int nb1 = comp(n0, m3(o0 + 1)), nb2 = comp(n0, m3(o0 + 2));
      M.tv[tri0] = make_int4(newp, p2, p0, 0);
      M.tv[tri1] = make_int4(newp, p1, p2, 0);
      if (tri2 == -1) {
        M.tn[tri0] = make_int4(nb2, -1, (tri1 << 2) | 1, 0);
        M.tn[tri1] = make_int4(nb1, (tri0 << 2) | 2, -1, 0);
      } else {
        M.tn[tri0] = make_int4(nb2, (tri2 << 2) | 2, (tri1 << 2) | 1, 0);
        M.tn[tri1] = make_int4(nb1, (tri0 << 2) | 2, (tri3 << 2) | 1, 0);
      }
      M.tst[tri0] |= TS_CHECK;
      M.tflip[tri0] = 1;
      M.tfo[tri0] = 0;
      M.tst[tri1] = TS_NOTNULL | TS_CHECK;
      M.tflip[tri1] = 1;
      M.tfo[tri1] = 0;
      if (tri2 != -1) {
        int4 v2 = M.tv[tri2], n2 = M.tn[tri2], s2 = M.tsg[tri2];
        int q0 = comp(v2, m3(o1 + 1)), q1 = comp(v2, m3(o1 + 2)), q2 = comp(v2, o1);
        int sg2[3] = {comp(s2, o1), comp(s2, m3(o1 + 1)), comp(s2, m3(o1 + 2))};
        M.tsg[tri2] = make_int4(sg2[1], -1, sg2[0], 0);
        M.tsg[tri3] = make_int4(sg2[2], sg2[0], -1, 0);
        if (sg2[1] != -1) s2t_store(M, sg2[1], (tri2 << 2) | 0, epoch, wkey(pos, 5));
        if (sg2[2] != -1) s2t_store(M, sg2[2], (tri3 << 2) | 0, epoch, wkey(pos, 6));
        int m1 = comp(n2, m3(o1 + 1)), m2 = comp(n2, m3(o1 + 2));
        M.tv[tri2] = make_int4(newp, q1, q2, 0);
        M.tn[tri2] = make_int4(m1, (tri3 << 2) | 2, (tri0 << 2) | 1, 0);
        M.tv[tri3] = make_int4(newp, q2, q0, 0);
        M.tn[tri3] = make_int4(m2, (tri1 << 2) | 2, (tri2 << 2) | 1, 0);
        M.tst[tri2] |= TS_CHECK;
        M.tflip[tri2] = 1;
        M.tfo[tri2] = 0;
        M.tst[tri3] = TS_NOTNULL | TS_CHECK;
        M.tflip[tri3] = 1;
        M.tfo[tri3] = 0;
      }
    }
    count_event(counter);
  }
}

// kernelUpdateSteinerNeighbors, refine.cu:4902-5059
GQM_KERNEL void k_update_steiner_nbrs(Mesh M, const int *wl, const int *dn, const int *sinks) {
  int n = *dn;
  GS_LOOP(pos, n) {
    int tindex = wl[pos];
    int index = sinks[tindex] >> 2, direction = sinks[tindex] & 3;
    if (direction != 3 && M.tfo[index] == 15) continue;
    int tri[4], iteration;
    int4 n0 = M.tn[index];
    tri[0] = index;
    if (direction == 3) {
      iteration = 3;
      tri[1] = dtri(n0.y);
      tri[2] = dtri(n0.z);
    } else {
      tri[1] = dtri(n0.z);
      if (n0.y == -1)
        iteration = 2;
      else {
        iteration = 4;
        tri[2] = dtri(n0.y);
        tri[3] = dtri(ld1(M.tn, tri[1], 2));
      }
    }
    relink_outer(M, tri, iteration);
  }
}

// kernelUpdateSteinerOnsegs, refine.cu:5091-5105 (over all subsegments)
template <class N>
GQM_KERNEL void k_onsegs_to_enc(Mesh M, const int *encl2, N ns_) {
  const int ns = nval(ns_);
  GS_LOOP(s, ns) if (encl2[s] >= 0) M.enc[s] = 1;
}

// ============================================================================
// Output compaction (refine.cu:5758-6484)
// ============================================================================
GQM_KERNEL void k_compact_tris_move(Mesh M, const int *tail, const int *empty, const int *dn, int *newidx) {
  int n = *dn;
  GS_LOOP(k, n) {
    int from = tail[k], to = empty[k];
    M.tv[to] = M.tv[from];
    M.tn[to] = M.tn[from];
    M.tst[to] = M.tst[from];
    M.tflip[to] = M.tflip[from];
    M.tfo[to] = M.tfo[from];
    newidx[from] = to;
  }
}
GQM_KERNEL void k_newidx_init(const Mesh M, int *newidx, int n, int newn, const uint8_t *flag, uint8_t deadbit,
                              bool dead_when_set) {
  GS_LOOP(i, n) {
    bool dead = dead_when_set ? (flag[i] & deadbit) != 0 : (flag[i] & deadbit) == 0;
    newidx[i] = dead ? -1 : (i < newn ? i : -2);
  }
}
GQM_KERNEL void k_fix_nbrs(Mesh M, const int *newidx, int newn) {
  GS_LOOP(t, newn) {
    int4 nb = M.tn[t];
    if (nb.x >= 0) nb.x = etri(newidx[dtri(nb.x)], dori(nb.x));
    if (nb.y >= 0) nb.y = etri(newidx[dtri(nb.y)], dori(nb.y));
    if (nb.z >= 0) nb.z = etri(newidx[dtri(nb.z)], dori(nb.z));
    M.tn[t] = nb;
  }
}
GQM_KERNEL void k_fix_s2t(Mesh M, const int *newidx, int ns) {
  GS_LOOP(s, ns) {
    int o = s2t_get(M, s);
    if (o >= 0) M.s2t[s] = s2t_plain(etri(newidx[dtri(o)], dori(o)));
  }
}
GQM_KERNEL void k_compact_pts_move(Mesh M, const int *tail, const int *empty, const int *dn, int *newidx) {
  int n = *dn;
  GS_LOOP(k, n) {
    int from = tail[k], to = empty[k];
    M.pts[to] = M.pts[from];
    M.ps[to] = M.ps[from];
    M.pred[to] = M.pred[from];
    newidx[from] = to;
  }
}
GQM_KERNEL void k_fix_tri_vertices(Mesh M, const int *newidx, int nt) {
  GS_LOOP(t, nt) {
    int4 v = M.tv[t];
    v.x = newidx[v.x];
    v.y = newidx[v.y];
    v.z = newidx[v.z];
    M.tv[t] = v;
  }
}
// plain output arrays (trianglelist, neighborlist via decode, segmentlist)
GQM_KERNEL void k_emit_output(Mesh M, int nt, int ns, int *tri, int *nbr, int *seg, uint8_t *tstat) {
  GS_LOOP(i, max(nt, ns)) {
    if (i < nt) {
      int4 v = M.tv[i], nb = M.tn[i];
      tri[3 * i] = v.x;
      tri[3 * i + 1] = v.y;
      tri[3 * i + 2] = v.z;
      nbr[3 * i] = dtri(nb.x);
      nbr[3 * i + 1] = dtri(nb.y);
      nbr[3 * i + 2] = dtri(nb.z);
      tstat[i] = (uint8_t)((M.tst[i] & 7) | (M.tflip[i] ? 8 : 0) | (M.tfo[i] << 4));
    }
    if (i < ns) {
      int o = s2t_get(M, i);
      if (o < 0) {
        seg[2 * i] = seg[2 * i + 1] = -1;
      } else {
        int t = dtri(o), r = dori(o);
        int4 v = M.tv[t];
        seg[2 * i] = comp(v, m3(r + 1));
        seg[2 * i + 1] = comp(v, m3(r + 2));
      }
    }
  }
}
GQM_KERNEL void k_emit_pstatus(Mesh M, int np, uint8_t *pstat) {
  GS_LOOP(i, np) pstat[i] = (uint8_t)((M.ps[i] & 15) | (M.pred[i] ? 16 : 0));
}

// ---------------------------------------------------------------------------
// The placement step and the collection of training data
// ---------------------------------------------------------------------------
#ifdef GQM_CTA_MODE
#define GQM_BID 0
#define GQM_NB 1
#else
#define GQM_BID ((int)blockIdx.x)
#define GQM_NB ((int)gridDim.x)
#endif

// Learned placement over the bad triangles, after k_circumcenter has written
// the plain centers: up to kInferWarpsMax warps per block, 32 candidates per
// warp and pass, the network's weights staged in the block's shared memory.
// ctr[0] counts candidates, ctr[1] the points the network placed.
GQM_KERNEL void k_learned_place(Mesh M, const int *bad, const int *dn, MlpDev P, double2 *center,
                                unsigned long long *ctr) {
#ifdef GQM_HOST_EMU
  const int n = *dn;
  for (int k = 0; k < n; ++k) {
    const int t = bad[k];
    const int4 v = M.tv[t];
    const double2 coff = center[k];
    const double2 cc = circumcenter(M.pts[v.x], M.pts[v.y], M.pts[v.z], 0.0, false);
    if (coff.x == cc.x && coff.y == cc.y) continue;
    float f[kFeat];
    features_of(M, t, bisector_of(M, t), 0.0, f);
    const float y = mlp_forward_row(P, f);
    ctr[0]++;
    if (y > 0.0f && y < 1.0f) {
      const double2 p = make_double2(coff.x + (double)y * (cc.x - coff.x), coff.y + (double)y * (cc.y - coff.y));
      if (!encroaches_near(M, t, p)) {
        center[k] = p;
        ctr[1]++;
      }
    }
  }
#else
  __shared__ MlpInferTiles sm;
  mlp_stage(P, sm.w);
  __syncthreads();
  const int warp = (int)(threadIdx.x >> 5), lane = (int)(threadIdx.x & 31u);
  const int nw = min(kInferWarpsMax, (int)(blockDim.x >> 5));
  if (warp >= nw) return;
  uint16_t *x = sm.x[warp];
  const int n = *dn;
  for (int g0 = (GQM_BID * nw + warp) * 32; g0 < n; g0 += GQM_NB * nw * 32) {
    const int k = g0 + lane;
    bool cand = false;
    int t = -1;
    double2 coff = make_double2(0.0, 0.0), cc = coff;
    if (k < n) {
      t = bad[k];
      const int4 v = M.tv[t];
      coff = center[k];
      cc = circumcenter(M.pts[v.x], M.pts[v.y], M.pts[v.z], 0.0, false);
      cand = (coff.x != cc.x || coff.y != cc.y);
    }
    const unsigned m = __ballot_sync(0xffffffffu, cand);
    if (!m) continue;
    float f[kFeat];
    if (cand) {
      const Bisector B = bisector_of(M, t);
      features_of(M, t, B, 0.0, f);
    } else {
      for (int j = 0; j < kFeat; ++j) f[j] = 0.0f;
    }
    mlp_put_row(x, lane, f);
    __syncwarp();
    const float y = mlp_forward_regs(sm.w, x);
    __syncwarp();
    bool used = false;
    if (cand && y > 0.0f && y < 1.0f) {
      const double2 p = make_double2(coff.x + (double)y * (cc.x - coff.x), coff.y + (double)y * (cc.y - coff.y));
      if (!encroaches_near(M, t, p)) {
        center[k] = p;
        used = true;
      }
    }
    const unsigned u = __ballot_sync(0xffffffffu, used);
    if (lane == 0) {
      atomicAdd(ctr, (unsigned long long)__popc(m));
      atomicAdd(ctr + 1, (unsigned long long)__popc(u));
    }
  }
#endif
}

// Number of triangles with an angle below theta among those that point c
// would form with the boundary of its Delaunay cavity (the triangles whose
// circumcircle contains c, reached from t0 without crossing a subsegment);
// 100 when the cavity has more than 64 triangles.
__device__ inline int star_bad_count(const Mesh &M, int t0, double2 c) {
  int list[64];
  int n = 0, nbad = 0;
  list[n++] = t0;
  for (int i = 0; i < n; ++i) {
    const int tri = list[i];
    const int4 v = M.tv[tri], nb = M.tn[tri], sg = M.tsg[tri];
    const int vv[3] = {v.x, v.y, v.z};
    for (int e = 0; e < 3; ++e) {
      bool boundary = comp(sg, e) >= 0 || comp(nb, e) < 0;
      if (!boundary) {
        const int nt = dtri(comp(nb, e));
        bool seen = false;
        for (int j = 0; j < n && !seen; ++j) seen = (list[j] == nt);
        if (seen) continue;
        const int4 w = M.tv[nt];
        const double2 a = M.pts[w.x], b = M.pts[w.y], d = M.pts[w.z];
        if (gqm_incircle_det_ref(a.x, a.y, b.x, b.y, d.x, d.y, c.x, c.y) > 0.0) {
          if (n == 64) return 100;
          list[n++] = nt;
          continue;
        }
        boundary = true;
      }
      // star triangle (c, u, w) on the boundary edge
      const double2 u = M.pts[vv[(e + 1) % 3]], w = M.pts[vv[(e + 2) % 3]];
      const double l0 = (u.x - w.x) * (u.x - w.x) + (u.y - w.y) * (u.y - w.y);
      const double l1 = (c.x - w.x) * (c.x - w.x) + (c.y - w.y) * (c.y - w.y);
      const double l2 = (c.x - u.x) * (c.x - u.x) + (c.y - u.y) * (c.y - u.y);
      // smallest angle is opposite the shortest side: cos^2 by the law of cosines
      double a2 = l0, b2 = l1, c2 = l2;
      if (b2 < a2) { const double tt = a2; a2 = b2; b2 = tt; }
      if (c2 < a2) { const double tt = a2; a2 = c2; c2 = tt; }
      const double num = b2 + c2 - a2;
      const double cos2 = (num * num) / (4.0 * b2 * c2);
      if (num > 0.0 && cos2 > M.gc2) nbad++;
    }
  }
  return nbad;
}

// Training rows: features and target t of every learned-placement candidate
// among the bad triangles (centers hold the plain points).
GQM_KERNEL void k_collect(Mesh M, const int *bad, const int *dn, const double2 *center, float *feat, float *target,
                          unsigned long long *count, unsigned long long cap) {
  const int n = *dn;
  GS_LOOP(k, n) {
    const int t = bad[k];
    const int4 v = M.tv[t];
    const double2 coff = center[k];
    const double2 cc = circumcenter(M.pts[v.x], M.pts[v.y], M.pts[v.z], 0.0, false);
    if (coff.x == cc.x && coff.y == cc.y) continue;
    int best = 1 << 30, bj = 0;
    for (int j = 0; j <= 8; ++j) {
      const double tj = j / 8.0;
      const double2 p = make_double2(coff.x + tj * (cc.x - coff.x), coff.y + tj * (cc.y - coff.y));
      if (j > 0 && encroaches_near(M, t, p)) continue;
      const int c = star_bad_count(M, t, p);
      if (c < best) {  // a point beyond the off-center only when it is strictly better
        best = c;
        bj = j;
      }
    }
    const unsigned long long row = atomicAdd(count, 1ull);
    if (row >= cap) continue;
    const Bisector B = bisector_of(M, t);
    features_of(M, t, B, 0.0, feat + row * kFeat);
    target[row] = bj / 8.0f;
  }
}

// ---------------------------------------------------------------------------
// Exploration runs for descendant-count labels (gqm_learn_explore).  Every
// bad triangle's candidate gets one row; the candidate inserts its point at
// t = j / (levels - 1) of the way from the off-center to the circumcenter, j
// drawn from a seeded hash of the triangle's vertices.  Lineage: every vertex
// inserted during the run carries the row of the candidate it descends from
// (vrow); a candidate's parent is the youngest such row among its bad
// triangle's vertices (the vertex whose insertion, directly or through the
// flips that followed it, made the triangle), and a midpoint descends from the
// youngest row among the vertices of the two triangles on its subsegment (the
// encroaching vertex is the apex of one of them).
// ---------------------------------------------------------------------------
struct ExploreDev {
  float *feat;     // [cap][kFeat]
  int *level;      // level j drawn (-1: off-center and circumcenter coincide)
  float *tused;    // t of the inserted point (0 when the drawn point would encroach)
  int *parent;     // parent row or -1
  uint8_t *ins;    // 1 once the candidate's point is in the mesh
  int *mids;       // midpoints that descend from the row directly
  unsigned long long *cnt;
  unsigned long long cap;
  int *vrow;       // per vertex slot: row it descends from (-1: input vertex)
  int *crow;       // per bad-list position: the candidate's row (-1: beyond cap)
  int *mlin;       // per midpoint position: its lineage, between the two kernels around k_insert_mid
  int levels;
  unsigned seed;
  // exploration around a network: with probability 1 - eps (per triangle,
  // from the same hash) the candidate takes the network's t (level -2)
  MlpDev net;
  int use_net;
  float eps;
};

// murmur3's 32-bit finaliser over the seed and the sorted vertex ids
__device__ __forceinline__ unsigned explore_mix(unsigned h) {
  h ^= h >> 16;
  h *= 0x85ebca6bu;
  h ^= h >> 13;
  h *= 0xc2b2ae35u;
  h ^= h >> 16;
  return h;
}
__device__ __forceinline__ unsigned explore_draw(unsigned seed, int a, int b, int c) {
  int lo = min(a, min(b, c)), hi = max(a, max(b, c)), mid = a + b + c - lo - hi;
  unsigned h = explore_mix(seed ^ 0x9e3779b9u);
  h = explore_mix(h ^ (unsigned)lo);
  h = explore_mix(h ^ (unsigned)mid);
  return explore_mix(h ^ (unsigned)hi);
}
__device__ __forceinline__ int explore_youngest(const int *vrow, int4 v) {
  return max(vrow[v.x], max(vrow[v.y], vrow[v.z]));
}

// after k_circumcenter: rows of the candidates, the drawn points into center
GQM_KERNEL void k_explore_place(Mesh M, const int *bad, const int *dn, double2 *center, ExploreDev E) {
  const int n = *dn;
  GS_LOOP(k, n) {
    const int t = bad[k];
    const int4 v = M.tv[t];
    const double2 coff = center[k];
    const double2 cc = circumcenter(M.pts[v.x], M.pts[v.y], M.pts[v.z], 0.0, false);
    const bool cand = (coff.x != cc.x || coff.y != cc.y);
    float f[kFeat];
    for (int q = 0; q < kFeat; ++q) f[q] = 0.0f;
    if (cand) features_of(M, t, bisector_of(M, t), 0.0, f);
    int j = -1;
    float tu = 0.0f;
    if (cand) {
      const unsigned h = explore_draw(E.seed, v.x, v.y, v.z);
      double tj = 0.0;
      if (E.use_net && (float)(explore_mix(h) >> 8) * (1.0f / 16777216.0f) >= E.eps) {
        j = -2;
        const float y = mlp_forward_row(E.net, f);
        tj = (y > 0.0f && y < 1.0f) ? (double)y : 0.0;
      } else {
        j = (int)(h % (unsigned)E.levels);
        tj = (double)j / (double)(E.levels - 1);
      }
      if (tj > 0.0) {
        const double2 p = make_double2(coff.x + tj * (cc.x - coff.x), coff.y + tj * (cc.y - coff.y));
        if (!encroaches_near(M, t, p)) {
          center[k] = p;
          tu = (float)tj;
        }
      }
    }
    const unsigned long long row = atomicAdd(E.cnt, 1ull);
    E.crow[k] = row < E.cap ? (int)row : -1;
    if (row >= E.cap) continue;
    for (int q = 0; q < kFeat; ++q) E.feat[row * kFeat + q] = f[q];
    E.level[row] = j;
    E.tused[row] = tu;
    E.parent[row] = explore_youngest(E.vrow, v);
    E.ins[row] = 0;
    E.mids[row] = 0;
  }
}

// after k_insert_steiner: the inserted points take their candidates' rows
// (a winner on a subsegment is not inserted and leaves its slot deleted)
template <class S>
GQM_KERNEL void k_explore_steiner(Mesh M, const int *wl, const int *dn, const double2 *center, S pslots_,
                                  ExploreDev E) {
  const int *pslots = slots_of(pslots_);
  const int n = *dn;
  GS_LOOP(pos, n) {
    const int k = wl[pos];
    const int newp = pslots[pos];
    if (M.ps[newp] != (PS_STEINER | PS_NEW)) continue;
    const double2 p = M.pts[newp], c = center[k];
    if (p.x != c.x || p.y != c.y) continue;
    const int row = E.crow[k];
    E.vrow[newp] = row;
    if (row >= 0) E.ins[row] = 1;
  }
}

// after k_mid_snapshot, before k_insert_mid: each midpoint's lineage
GQM_KERNEL void k_explore_mid_pre(Mesh M, const int *dn, const int *snap, ExploreDev E) {
  const int n = *dn;
  GS_LOOP(pos, n) {
    const int otri = snap[pos];
    const int t0 = dtri(otri);
    int lin = -1;
    if (t0 >= 0) {
      lin = explore_youngest(E.vrow, M.tv[t0]);
      const int on = ld1(M.tn, t0, dori(otri));
      if (on >= 0) lin = max(lin, explore_youngest(E.vrow, M.tv[dtri(on)]));
    }
    E.mlin[pos] = lin;
  }
}

// after k_insert_mid: the inserted midpoints take their lineage
template <class S>
GQM_KERNEL void k_explore_mid_post(Mesh M, const int *mids, const int *dn, S pslots_, ExploreDev E) {
  const int *pslots = slots_of(pslots_);
  const int n = *dn;
  GS_LOOP(pos, n) {
    const int newp = pslots[mids[pos]];
    if (M.ps[newp] != (PS_STEINER | PS_NEW | PS_SEGSPLIT)) continue;
    const int lin = E.mlin[pos];
    E.vrow[newp] = lin;
    if (lin >= 0) atomicAdd(E.mids + lin, 1);
  }
}

}  // namespace gqm
