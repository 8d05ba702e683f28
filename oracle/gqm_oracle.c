/* Test oracle: plain-C restatement of the reference's GPU quality refinement
 * (GPU_Refine/refine.cu).  Test infrastructure only; see gqm_oracle.h.
 *
 * Execution model.  Each reference kernel is emulated by a loop over its
 * thread positions in ascending order, on the state the previous kernel left.
 * Thrust stream compactions become ordered scans.  Host bookkeeping (free-slot
 * lists, growth by blocks, high-water marks) is reproduced exactly, because
 * slot numbers decide every conflict (atomicMin on indices).
 *
 * Arithmetic.  Built with -ffp-contract=off: every FP64 operation is rounded
 * on its own, which matches the reference compiled with nvcc -fmad=false.
 * Built with -DGQM_ORACLE_CONTRACTED=1 (libgqm_oracle_fma.so), madd() fuses
 * the products that the reference as its project builds it (nvcc's default
 * contraction) fuses, one rounding for the product and the add; which
 * products those are was measured on the reference's compiled kernels and
 * predicates, by comparing their outputs with every candidate evaluation.
 * The reference's device predicate constants are never initialised
 * (GPU_Refine/cudaCCW.h:41), so orientation is the plain determinant and
 * incircle falls back to an expansion with a zero splitter only when the plain
 * determinant is exactly zero; both are restated below.
 *
 * Races in the reference and the rule used here (shared with the CUDA code):
 *  R1 kernelCheckFlipping reads a neighbour's flip flag (refine.cu:831) that
 *     the neighbour's own thread may clear (refine.cu:1069).  Rule: the flag
 *     is read as it was when the kernel started.
 *  R3 kernelInsertMidPoints reads subseg2tri[sindex] (refine.cu:2636) while
 *     a winning thread may rewrite that entry (2848-2850) when the subsegment
 *     is an outer edge of the winner's triangles.  Rule: the entry is read as
 *     it was when the kernel started, so such a thread loses as intended.
 *  R2 Two threads of one kernel may store different orientations into the
 *     same subseg2tri entry (a subsegment whose two sides belong to two
 *     different winners: refine.cu:1362-1372, 1419-1424, 1533-1544,
 *     2844-2850, 2900-2903, 4744-4749, 4814-4817, 4873-4876).  Rule: within
 *     one kernel launch, the store that lands is decided by the storing
 *     threads' warps and lanes and the stores' program order (wkey below).
 *  Everything else the reference does concurrently is order independent.
 *
 * Deliberate difference: initSubsegs (refine.cu:5691-5747) does not reset
 * `scanfinish` between chunks of 1,280,000 triangles and indexes the output
 * with `pos` instead of `pos + trioffset` (refine.cu:5667-5681), so inputs
 * with more triangles are mishandled.  This restatement matches every
 * triangle against every segment, which is what the reference computes for
 * inputs of up to 1,280,000 triangles.
 */
#include "gqm_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define PI_REF 3.141592653589793238462643383279502884197169399375105820974944592308
#define MAXINT_REF 2147483647
#define LS_REF 50

/* ---------------- status bits (refine.h:36-205) ---------------- */
#define PS_DELETED 1
#define PS_STEINER 2
#define PS_SEGSPLIT 4
#define PS_NEW 8
#define PS_REDUNDANT 16

#define TS_NOTNULL 1
#define TS_BAD 2
#define TS_CHECK 4
#define TS_FLIP 8

static inline int ts_null(unsigned char s) { return (s & TS_NOTNULL) == 0; }
static inline int ts_flipori(unsigned char s) { return (s >> 4) & 15; }
static inline void ts_setflipori(unsigned char *s, int o) { *s = (unsigned char)((*s & 0x0f) | (o << 4)); }
static inline void ts_set(unsigned char *s, int bit, int on) {
  if (on)
    *s |= (unsigned char)bit;
  else
    *s &= (unsigned char)~bit;
}

/* ---------------- oriented triangles (refine.cu:95-113) ---------------- */
static inline int dtri(int t) { return t >= 0 ? (t >> 2) : -1; }
static inline int dori(int t) { return t & 3; }
static inline int etri(int t, int o) { return t >= 0 ? ((t << 2) | o) : -1; }
static inline int negate_ref(int i) { return -i - 3; }

typedef struct {
  double x, y;
} P2;

#ifndef GQM_ORACLE_CONTRACTED
#define GQM_ORACLE_CONTRACTED 0
#endif
/* a * b + c: fused where the reference's contracted build fuses, else two roundings */
static inline double madd(double a, double b, double c) {
#if GQM_ORACLE_CONTRACTED
  return fma(a, b, c);
#else
  return a * b + c;
#endif
}

/* ---------------- predicates (cudaCCW.h with zero constants) ---------------- */
static double orient_ref(P2 a, P2 b, P2 c) {
  double detleft = (a.x - c.x) * (b.y - c.y);
  double detright = (a.y - c.y) * (b.x - c.x);
  return detleft - detright;
}

static double incircle_det(P2 a, P2 b, P2 c, P2 d) {
  double adx = a.x - d.x, bdx = b.x - d.x, cdx = c.x - d.x;
  double ady = a.y - d.y, bdy = b.y - d.y, cdy = c.y - d.y;
  double bdxcdy = bdx * cdy, cdxbdy = cdx * bdy;
  double alift = madd(adx, adx, ady * ady);
  double cdxady = cdx * ady, adxcdy = adx * cdy;
  double blift = madd(bdx, bdx, bdy * bdy);
  double adxbdy = adx * bdy, bdxady = bdx * ady;
  double clift = madd(cdx, cdx, cdy * cdy);
  return madd(clift, adxbdy - bdxady, madd(alift, bdxcdy - cdxbdy, blift * (cdxady - adxcdy)));
}

/* error-free transforms, cudaCCW.h:89-176 */
static void o_two_sum(double a, double b, double *x, double *y) {
  double s = a + b, bv = s - a, av = s - bv, br = b - bv, ar = a - av;
  *x = s;
  *y = ar + br;
}
static void o_two_diff(double a, double b, double *x, double *y) {
  double s = a - b, bv = a - s, av = s + bv, br = bv - b, ar = a - av;
  *x = s;
  *y = ar + br;
}
static void o_fast_two_sum(double a, double b, double *x, double *y) {
  double s = a + b, bv = s - a;
  *x = s;
  *y = b - bv;
}
/* Two_Product with splitter constData[0] == 0 */
static void o_two_product(double a, double b, double *x, double *y) {
  double p = a * b;
  double c = 0.0 * a, abig = c - a, ahi = c - abig, alo = a - ahi;
  double cb = 0.0 * b, bbig = cb - b, bhi = cb - bbig, blo = b - bhi;
  double e1 = p - (ahi * bhi), e2 = e1 - (alo * bhi), e3 = e2 - (ahi * blo);
  *x = p;
  *y = (alo * blo) - e3;
}
static void o_two_two_diff(double a1, double a0, double b1, double b0, double *r) {
  double i, j, z, t;
  o_two_diff(a0, b0, &i, &r[0]);
  o_two_sum(a1, i, &j, &z);
  o_two_diff(z, b1, &i, &r[1]);
  o_two_sum(j, i, &r[3], &t);
  r[2] = t;
}
static int o_fes(int elen, const double *e, int flen, const double *f, double *h) {
  double Q, Qn, hh, en = e[0], fn = f[0];
  int ei = 0, fi = 0, hi = 0;
  if ((fn > en) == (fn > -en)) {
    Q = en;
    ++ei;
    en = ei < elen ? e[ei] : 0.0;
  } else {
    Q = fn;
    ++fi;
    fn = fi < flen ? f[fi] : 0.0;
  }
  if (ei < elen && fi < flen) {
    if ((fn > en) == (fn > -en)) {
      o_fast_two_sum(en, Q, &Qn, &hh);
      ++ei;
      en = ei < elen ? e[ei] : 0.0;
    } else {
      o_fast_two_sum(fn, Q, &Qn, &hh);
      ++fi;
      fn = fi < flen ? f[fi] : 0.0;
    }
    Q = Qn;
    if (hh != 0.0) h[hi++] = hh;
    while (ei < elen && fi < flen) {
      if ((fn > en) == (fn > -en)) {
        o_two_sum(Q, en, &Qn, &hh);
        ++ei;
        en = ei < elen ? e[ei] : 0.0;
      } else {
        o_two_sum(Q, fn, &Qn, &hh);
        ++fi;
        fn = fi < flen ? f[fi] : 0.0;
      }
      Q = Qn;
      if (hh != 0.0) h[hi++] = hh;
    }
  }
  while (ei < elen) {
    o_two_sum(Q, en, &Qn, &hh);
    ++ei;
    en = ei < elen ? e[ei] : 0.0;
    Q = Qn;
    if (hh != 0.0) h[hi++] = hh;
  }
  while (fi < flen) {
    o_two_sum(Q, fn, &Qn, &hh);
    ++fi;
    fn = fi < flen ? f[fi] : 0.0;
    Q = Qn;
    if (hh != 0.0) h[hi++] = hh;
  }
  if (Q != 0.0 || hi == 0) h[hi++] = Q;
  return hi;
}
static int o_scale(int elen, const double *e, double b, double *h) {
  double Q, sum, hh, p1, p0;
  int hi = 0;
  o_two_product(e[0], b, &Q, &hh);
  if (hh != 0) h[hi++] = hh;
  for (int i = 1; i < elen; i++) {
    o_two_product(e[i], b, &p1, &p0);
    o_two_sum(Q, p0, &sum, &hh);
    if (hh != 0) h[hi++] = hh;
    o_fast_two_sum(p1, sum, &Q, &hh);
    if (hh != 0) h[hi++] = hh;
  }
  if (Q != 0.0 || hi == 0) h[hi++] = Q;
  return hi;
}
/* cuda_incircleexact, cudaCCW.h:570-666 */
static double incircle_expansion(P2 a, P2 b, P2 c, P2 d) {
  double x1, x0, y1, y0, ab[4], bc[4], cd[4], da[4], ac[4], bd[4], t8[8], abc[12], bcd[12], cda[12], dab[12];
  double d24x[24], d24y[24], d48x[48], d48y[48], ad[96], bdt[96], cdt[96], ddt[96], abd[192], cdd[192], det[384];
  int tl, abcl, bcdl, cdal, dabl, xl, yl, al, bl, cl, dl, abl, cdl, dtl;
  o_two_product(a.x, b.y, &x1, &x0);
  o_two_product(b.x, a.y, &y1, &y0);
  o_two_two_diff(x1, x0, y1, y0, ab);
  o_two_product(b.x, c.y, &x1, &x0);
  o_two_product(c.x, b.y, &y1, &y0);
  o_two_two_diff(x1, x0, y1, y0, bc);
  o_two_product(c.x, d.y, &x1, &x0);
  o_two_product(d.x, c.y, &y1, &y0);
  o_two_two_diff(x1, x0, y1, y0, cd);
  o_two_product(d.x, a.y, &x1, &x0);
  o_two_product(a.x, d.y, &y1, &y0);
  o_two_two_diff(x1, x0, y1, y0, da);
  o_two_product(a.x, c.y, &x1, &x0);
  o_two_product(c.x, a.y, &y1, &y0);
  o_two_two_diff(x1, x0, y1, y0, ac);
  o_two_product(b.x, d.y, &x1, &x0);
  o_two_product(d.x, b.y, &y1, &y0);
  o_two_two_diff(x1, x0, y1, y0, bd);
  tl = o_fes(4, cd, 4, da, t8);
  cdal = o_fes(tl, t8, 4, ac, cda);
  tl = o_fes(4, da, 4, ab, t8);
  dabl = o_fes(tl, t8, 4, bd, dab);
  for (int i = 0; i < 4; i++) {
    bd[i] = -bd[i];
    ac[i] = -ac[i];
  }
  tl = o_fes(4, ab, 4, bc, t8);
  abcl = o_fes(tl, t8, 4, ac, abc);
  tl = o_fes(4, bc, 4, cd, t8);
  bcdl = o_fes(tl, t8, 4, bd, bcd);
  xl = o_scale(bcdl, bcd, a.x, d24x);
  xl = o_scale(xl, d24x, a.x, d48x);
  yl = o_scale(bcdl, bcd, a.y, d24y);
  yl = o_scale(yl, d24y, a.y, d48y);
  al = o_fes(xl, d48x, yl, d48y, ad);
  xl = o_scale(cdal, cda, b.x, d24x);
  xl = o_scale(xl, d24x, -b.x, d48x);
  yl = o_scale(cdal, cda, b.y, d24y);
  yl = o_scale(yl, d24y, -b.y, d48y);
  bl = o_fes(xl, d48x, yl, d48y, bdt);
  xl = o_scale(dabl, dab, c.x, d24x);
  xl = o_scale(xl, d24x, c.x, d48x);
  yl = o_scale(dabl, dab, c.y, d24y);
  yl = o_scale(yl, d24y, c.y, d48y);
  cl = o_fes(xl, d48x, yl, d48y, cdt);
  xl = o_scale(abcl, abc, d.x, d24x);
  xl = o_scale(xl, d24x, -d.x, d48x);
  yl = o_scale(abcl, abc, d.y, d24y);
  yl = o_scale(yl, d24y, -d.y, d48y);
  dl = o_fes(xl, d48x, yl, d48y, ddt);
  abl = o_fes(al, ad, bl, bdt, abd);
  cdl = o_fes(cl, cdt, dl, ddt, cdd);
  dtl = o_fes(abl, abd, cdl, cdd, det);
  return det[dtl - 1];
}
/* cuda_inCircle (668-708): the plain determinant, 0 when it is 0 */
static double incircle_ref(P2 a, P2 b, P2 c, P2 d) { return incircle_det(a, b, c, d); }
/* cuda_inCircle_exact (711-757) */
static double incircle_ref_exact(P2 a, P2 b, P2 c, P2 d) {
  double det = incircle_det(a, b, c, d);
  if (det > 0 || -det > 0) return det > 0 ? 1.0 : -1.0;
  return incircle_expansion(a, b, c, d);
}
/* the "cuda_inCircle, and cuda_inCircle_exact when it returns 0" pattern */
static double incircle_pair(P2 a, P2 b, P2 c, P2 d) {
  double r = incircle_ref(a, b, c, d);
  if (r == 0) r = incircle_ref_exact(a, b, c, d);
  return r;
}

/* ---------------- geometry helpers ---------------- */
/* checkseg4encroach, refine.cu:115-139 */
static int encroached(P2 o, P2 d, P2 a, double goodcoss /* cos^2 */, int mode) {
  double dot = madd(o.x - a.x, d.x - a.x, (o.y - a.y) * (d.y - a.y));
  if (dot < 0.0) {
    if (mode || dot * dot >= (2.0 * goodcoss - 1.0) * (2.0 * goodcoss - 1.0) *
                                   madd(o.x - a.x, o.x - a.x, (o.y - a.y) * (o.y - a.y)) *
                                   madd(d.x - a.x, d.x - a.x, (d.y - a.y) * (d.y - a.y)))
      return 1;
  }
  return 0;
}

/* kernelComputeSmallestAngle, refine.cu:317-374 */
static double smallest_angle(P2 pApex, P2 pOrg, P2 pDest, int *shortestOri) {
  double dxod = pOrg.x - pDest.x, dyod = pOrg.y - pDest.y;
  double dxda = pDest.x - pApex.x, dyda = pDest.y - pApex.y;
  double dxao = pApex.x - pOrg.x, dyao = pApex.y - pOrg.y;
  double lenOrg = madd(dyod, dyod, dxod * dxod), lenDest = madd(dyda, dyda, dxda * dxda);
  double lenApex = madd(dxao, dxao, dyao * dyao);
  double ang, sh;
  if (lenOrg < lenDest && lenOrg < lenApex) {
    sh = lenOrg;
    *shortestOri = 0;
    ang = madd(dyda, dyao, dxda * dxao);
  } else if (lenDest < lenOrg && lenDest < lenApex) {
    sh = lenDest;
    *shortestOri = 1;
    ang = madd(dyod, dyao, dxod * dxao);
  } else {
    sh = lenApex;
    *shortestOri = 2;
    ang = madd(dyod, dyda, dxod * dxda);
  }
  return ang * ang * sh / (lenOrg * lenDest * lenApex);
}

/* computeCircumcenter, refine.cu:3780-3868 */
static P2 circumcenter(P2 vApex, P2 vOrg, P2 vDest, double offConstant, int offcenter) {
  double xdo = vDest.x - vOrg.x, ydo = vDest.y - vOrg.y;
  double xao = vApex.x - vOrg.x, yao = vApex.y - vOrg.y;
  double dodist = madd(xdo, xdo, ydo * ydo);
  double aodist = madd(xao, xao, yao * yao);
  double dadist = madd(vDest.x - vApex.x, vDest.x - vApex.x, (vDest.y - vApex.y) * (vDest.y - vApex.y));
  double denominator;
  double tmp = xdo * yao - xao * ydo;
  if (tmp != 0)
    denominator = 0.5 / tmp;
  else
    denominator = 0.5 / orient_ref(vDest, vApex, vOrg);
  double dx = madd(yao, dodist, -(ydo * aodist)) * denominator;
  double dy = madd(xdo, aodist, -(xao * dodist)) * denominator;
  if (offcenter && (offConstant > 0.0)) {
    double dxoff, dyoff;
    if ((dodist < aodist) && (dodist < dadist)) {
      dxoff = 0.5 * xdo - offConstant * ydo;
      dyoff = madd(offConstant, xdo, 0.5 * ydo);
      if (madd(dxoff, dxoff, dyoff * dyoff) < madd(dx, dx, dy * dy)) {
        dx = dxoff;
        dy = dyoff;
      }
    } else if (aodist < dadist) {
      dxoff = 0.5 * xao + offConstant * yao;
      dyoff = 0.5 * yao - offConstant * xao;
      if (madd(dxoff, dxoff, dyoff * dyoff) < madd(dx, dx, dy * dy)) {
        dx = dxoff;
        dy = dyoff;
      }
    } else {
      dxoff = 0.5 * (vApex.x - vDest.x) - offConstant * (vApex.y - vDest.y);
      dyoff = madd(offConstant, vApex.x - vDest.x, 0.5 * (vApex.y - vDest.y));
      if (madd(dxoff, dxoff, dyoff * dyoff) < madd(dx - xdo, dx - xdo, (dy - ydo) * (dy - ydo))) {
        dx = xdo + dxoff;
        dy = ydo + dyoff;
      }
    }
  }
  P2 c;
  c.x = vOrg.x + dx;
  c.y = vOrg.y + dy;
  return c;
}

/* ---------------- growable int array ---------------- */
typedef struct {
  int *a;
  long n, cap;
} IV;
static void iv_reserve(IV *v, long n) {
  if (n > v->cap) {
    long c = v->cap ? v->cap : 16;
    while (c < n) c *= 2;
    v->a = (int *)realloc(v->a, sizeof(int) * c);
    v->cap = c;
  }
}
static void iv_resize(IV *v, long n, int fill) {
  iv_reserve(v, n);
  for (long i = v->n; i < n; ++i) v->a[i] = fill;
  v->n = n;
}
static void iv_push(IV *v, int x) {
  iv_reserve(v, v->n + 1);
  v->a[v->n++] = x;
}

/* ---------------- refinement state ---------------- */
typedef struct {
  /* capacities: PStatus.size() and TStatus.size() in the reference */
  long pcap, tcap;
  P2 *pts;
  unsigned char *ps;
  int *tri, *nbr, *t2s; /* 3 * tcap */
  unsigned char *ts;
  int *tmark;           /* t_trimarker, also the flipBy array, tcap */
  IV s2t, s2seg, enc;   /* per subsegment */
  unsigned *s2t_epoch;  /* rule R2: launch of the last store */
  unsigned *s2t_key;    /* rule R2: writer key of the last store (wkey) */
  long s2t_epoch_cap;
  unsigned epoch;
  int *segs;
  /* host bookkeeping */
  int last_point, last_triangle, last_subseg;
  int pointblock, triblock;
  int nempty_p, nempty_t;
  IV emptyp, emptyt;
  double theta, gc2;
  double max_area;  /* area bound (0: none), the counterpart of Triangle's `a` switch */
  int mode;
  long long max_rounds;
  int err;
  /* scratch */
  IV l0, l1, l2, l3, l4, l5;
  long long flip_steps, steiner_inserted, midpoints_inserted, bad_total;
} St;

static void s2t_begin(St *S) { S->epoch++; }
/* Key of one store to subseg2tri inside a launch (rule R2).  When several
 * threads of one launch store into the same subseg2tri entry, the store with
 * the largest key is the one kept, where the key orders the stores as the
 * reference's runs on a B200 were seen to land them:
 *   - two stores of one warp from different store instructions: the later
 *     instruction in program order lands last (a warp issues its stores in
 *     order);
 *   - two lanes of one store instruction: the lower lane's value is kept;
 *   - two different warps: the lower warp's store is kept.
 * Across warps the order is a race in the reference; this choice is the one
 * that the reference's own flip-step traces (tests/golden) follow on every
 * seeded configuration recorded there.  pos is the thread's position in the
 * launch, slot the store's place in the kernel's program order. */
static unsigned wkey(long pos, int slot) {
  return (unsigned)(((0x7FFFFFL - (pos >> 5)) << 9) | ((long)slot << 5) | (31 - (pos & 31)));
}
static void s2t_set(St *S, int s, int v, unsigned key) {
  if (s >= S->s2t_epoch_cap) {
    long c = S->s2t_epoch_cap ? S->s2t_epoch_cap : 64;
    while (c <= s) c *= 2;
    S->s2t_epoch = (unsigned *)realloc(S->s2t_epoch, sizeof(unsigned) * c);
    S->s2t_key = (unsigned *)realloc(S->s2t_key, sizeof(unsigned) * c);
    memset(S->s2t_epoch + S->s2t_epoch_cap, 0, sizeof(unsigned) * (c - S->s2t_epoch_cap));
    memset(S->s2t_key + S->s2t_epoch_cap, 0, sizeof(unsigned) * (c - S->s2t_epoch_cap));
    S->s2t_epoch_cap = c;
  }
  if (S->s2t_epoch[s] == S->epoch && S->s2t_key[s] > key) return;
  S->s2t.a[s] = v;
  S->s2t_epoch[s] = S->epoch;
  S->s2t_key[s] = key;
}

static void grow_points(St *S, long ncap) {
  S->pts = (P2 *)realloc(S->pts, sizeof(P2) * ncap);
  S->ps = (unsigned char *)realloc(S->ps, ncap);
  for (long i = S->pcap; i < ncap; ++i) {
    S->pts[i].x = S->pts[i].y = 0.0;
    S->ps[i] = PS_DELETED;
  }
  S->pcap = ncap;
}
static void grow_tris(St *S, long ncap) {
  S->tri = (int *)realloc(S->tri, sizeof(int) * 3 * ncap);
  S->nbr = (int *)realloc(S->nbr, sizeof(int) * 3 * ncap);
  S->t2s = (int *)realloc(S->t2s, sizeof(int) * 3 * ncap);
  S->ts = (unsigned char *)realloc(S->ts, ncap);
  S->tmark = (int *)realloc(S->tmark, sizeof(int) * ncap);
  for (long i = S->tcap; i < ncap; ++i) {
    S->tri[3 * i] = S->tri[3 * i + 1] = S->tri[3 * i + 2] = 0;
    S->nbr[3 * i] = S->nbr[3 * i + 1] = S->nbr[3 * i + 2] = 0;
    S->t2s[3 * i] = S->t2s[3 * i + 1] = S->t2s[3 * i + 2] = -1;
    S->ts[i] = 0;
    S->tmark[i] = 0;
  }
  S->tcap = ncap;
}

/* updateEmptyPoints / updateEmptyTriangles, refine.cu:149-197 */
static int refresh_empty_points(St *S) {
  S->emptyp.n = 0;
  for (long i = 0; i < S->pcap; ++i)
    if (S->ps[i] & PS_DELETED) iv_push(&S->emptyp, (int)i);
  return (int)S->emptyp.n;
}
static int refresh_empty_tris(St *S) {
  S->emptyt.n = 0;
  for (long i = 0; i < S->tcap; ++i)
    if (ts_null(S->ts[i])) iv_push(&S->emptyt, (int)i);
  return (int)S->emptyt.n;
}
/* the growth steps of refine.cu:3408-3444 and 5259-5296 */
static void ensure_slots(St *S, int npts, int ntris) {
  if (npts > S->nempty_p) {
    S->nempty_p = refresh_empty_points(S);
    int num = 0;
    while (npts > S->nempty_p + num * S->pointblock) num++;
    if (num != 0) {
      grow_points(S, S->pcap + (long)num * S->pointblock);
      S->nempty_p = refresh_empty_points(S);
    }
  }
  if (ntris > S->nempty_t) {
    S->nempty_t = refresh_empty_tris(S);
    int num = 0;
    while (ntris > S->nempty_t + num * S->triblock) num++;
    if (num != 0) {
      grow_tris(S, S->tcap + (long)num * S->triblock);
      S->nempty_t = refresh_empty_tris(S);
    }
  }
}
/* slot bookkeeping after an insertion batch, refine.cu:3545-3559, 5354-5368 */
static void consume_slots(St *S, int npts, int ntris) {
  int slot_after = (int)(S->pcap - S->last_point);
  int slot_before = S->nempty_p - slot_after;
  if (slot_before < npts) S->last_point += npts - slot_before;
  S->nempty_p -= npts;
  slot_after = (int)(S->tcap - S->last_triangle);
  slot_before = S->nempty_t - slot_after;
  if (slot_before < ntris) S->last_triangle += ntris - slot_before;
  S->nempty_t -= ntris;
}
static int new_point_slot(St *S, int k) { return S->emptyp.a[S->emptyp.n - S->nempty_p + k]; }
static int new_tri_slot(St *S, int k) { return S->emptyt.a[S->emptyt.n - S->nempty_t + k]; }

/* ---------------- flip-flop (refine.cu:580-2490) ---------------- */
/* markFan, refine.cu:580-602 */
static void mark_fan(St *S, int triIndex, int triOri) {
  int cur = triIndex, ori = triOri;
  long guard = 0;
  do {
    ts_set(&S->ts[cur], TS_FLIP, 1);
    int nx = S->nbr[cur * 3 + (ori + 2) % 3];
    cur = dtri(nx);
    ori = dori(nx);
    if (++guard > 4 * S->tcap + 16) {
      S->err = -4;
      return;
    }
  } while (cur > -1 && cur != triIndex);
}

static void compete(St *S, int index0, const int *others, int n, int code) {
  ts_setflipori(&S->ts[index0], code);
  if (index0 < S->tmark[index0]) S->tmark[index0] = index0;
  for (int k = 0; k < n; ++k)
    if (others[k] >= 0 && index0 < S->tmark[others[k]]) S->tmark[others[k]] = index0;
}
static void amin(int *a, int v) {
  if (v < *a) *a = v;
}

/* deleteOneFromTwo, refine.cu:733-757 */
static int delete_one_from_two(St *S, int pApex, int pOpp) {
  unsigned char a = S->ps[pApex], o = S->ps[pOpp];
  if ((a & PS_SEGSPLIT) && (o & PS_SEGSPLIT)) return -1;
  if ((a & PS_NEW) && (o & PS_NEW)) {
    if (a & PS_SEGSPLIT) return 1;
    if (o & PS_SEGSPLIT) return 0;
    return pApex < pOpp ? 1 : 0;
  }
  return -1;
}

/* kernelCheckFlipping thread body, refine.cu:778-1070; flip0 holds the flip
 * flags at kernel start (rule R1) */
static void check_flipping(St *S, int index, const unsigned char *flip0) {
  int *flipBy = S->tmark;
  int min = MAXINT_REF;
  int p[3] = {S->tri[index * 3], S->tri[index * 3 + 1], S->tri[index * 3 + 2]};
  for (int i = 0; i < 3; ++i)
    if ((S->ps[p[i]] & PS_REDUNDANT) && p[i] < min) min = p[i];
  P2 v[3] = {S->pts[p[0]], S->pts[p[1]], S->pts[p[2]]};
  for (int i = 0; i < 3; i++) {
    if (min == p[i]) continue;
    if (S->t2s[3 * index + i] != -1) continue;
    int tri = S->nbr[3 * index + i];
    int pTri = dtri(tri), pOri = dori(tri);
    if (index < pTri || (pTri >= 0 && !flip0[pTri])) {
      int pOpp = S->tri[pTri * 3 + pOri];
      if ((S->ps[pOpp] & PS_REDUNDANT) && pOpp < min) continue;
      P2 vOpp = S->pts[pOpp];
      int org = (i + 1) % 3, dest = (i + 2) % 3, apex = i;
      if (min != MAXINT_REF) {
        int deleteOri, n1, n2;
        if (min == p[org]) {
          deleteOri = (i + 2) % 3;
          n1 = S->nbr[index * 3 + dest];
          n2 = S->nbr[pTri * 3 + (pOri + 1) % 3];
        } else {
          deleteOri = i;
          n1 = S->nbr[index * 3 + org];
          n2 = S->nbr[pTri * 3 + (pOri + 2) % 3];
        }
        if (dtri(n1) == dtri(n2)) {
          int o[2] = {pTri, dtri(n1)};
          compete(S, index, o, 2, 3 + deleteOri);
          return;
        } else {
          int n1_tri = dtri(n1), n1_ori = dori(n1), n2_tri = dtri(n2), n2_ori = dori(n2);
          int n1_pOpp = S->tri[3 * n1_tri + n1_ori];
          int n2_pOpp = S->tri[3 * n2_tri + n2_ori];
          P2 n1_vOpp = S->pts[n1_pOpp], n2_vOpp = S->pts[n2_pOpp];
          int n3;
          if (min == p[org])
            n3 = S->nbr[3 * n1_tri + (n1_ori + 2) % 3];
          else
            n3 = S->nbr[3 * n1_tri + (n1_ori + 1) % 3];
          if (dtri(n3) == dtri(n2)) {
            if (min == p[org]) {
              double d = orient_ref(v[apex], v[org], vOpp);
              if (d == 0) {
                double t0 = orient_ref(v[dest], v[apex], n1_vOpp);
                double t1 = orient_ref(v[dest], v[org], n1_vOpp);
                int f0 = (t0 > 0 && t1 < 0);
                t0 = orient_ref(v[dest], v[org], n2_vOpp);
                t1 = orient_ref(v[dest], vOpp, n2_vOpp);
                int f1 = (t0 > 0 && t1 < 0);
                if (!f0 && !f1) {
                  if ((S->ps[n1_pOpp] & PS_REDUNDANT) && n1_pOpp < min) continue;
                  int o[3] = {pTri, n1_tri, n2_tri};
                  compete(S, index, o, 3, 6 + i);
                  return;
                }
              }
            } else {
              double d = orient_ref(v[apex], v[dest], vOpp);
              if (d == 0) {
                double t0 = orient_ref(v[org], v[dest], n1_vOpp);
                double t1 = orient_ref(v[org], v[apex], n1_vOpp);
                int f0 = (t0 > 0 && t1 < 0);
                t0 = orient_ref(v[org], vOpp, n2_vOpp);
                t1 = orient_ref(v[org], v[dest], n2_vOpp);
                int f1 = (t0 > 0 && t1 < 0);
                if (!f0 && !f1) {
                  if ((S->ps[n1_pOpp] & PS_REDUNDANT) && n1_pOpp < min) continue;
                  int o[3] = {pTri, n1_tri, n2_tri};
                  compete(S, index, o, 3, 6 + i);
                  return;
                }
              }
            }
          }
        }
        double t1 = orient_ref(v[apex], v[org], vOpp);
        if (t1 <= 0) continue;
        double t2 = orient_ref(v[apex], v[dest], vOpp);
        if (t2 >= 0) continue;
        {
          int o[1] = {pTri};
          compete(S, index, o, 1, (i + 2) % 3);
        }
        return;
      }
      double ret = incircle_pair(v[apex], v[org], v[dest], vOpp);
      double ret_opp = incircle_pair(v[org], vOpp, v[dest], v[apex]);
      double ret_after = incircle_pair(v[apex], v[org], vOpp, v[dest]);
      double ret_after_opp = incircle_pair(vOpp, v[dest], v[apex], v[org]);
      if (ret > 0 && ret_opp > 0 && ret_after < 0 && ret_after_opp < 0) {
        int td = delete_one_from_two(S, p[apex], pOpp);
        if (td == -1) {
          int o[1] = {pTri};
          compete(S, index, o, 1, (i + 2) % 3);
        } else if (td == 0) {
          amin(&flipBy[index], negate_ref(etri(index, (i + 2) % 3)));
        } else {
          int t = negate_ref(etri(pTri, (pOri + 2) % 3));
          amin(&flipBy[index], t);
          amin(&flipBy[pTri], t);
        }
        return;
      }
    }
  }
  ts_set(&S->ts[index], TS_FLIP, 0);
}

/* kernelMarkFlipWinner, refine.cu:1072-1170 */
static void mark_flip_winner(St *S, int index) {
  int *flipBy = S->tmark;
  int ori = ts_flipori(S->ts[index]);
  if (ori == 15) return;
  int win = 0;
  if (flipBy[index] == index) {
    if (ori < 3) {
      int pOppTri = dtri(S->nbr[index * 3 + (ori + 1) % 3]);
      if (flipBy[pOppTri] == index) win = 1;
    } else if (ori < 6) {
      ori -= 3;
      ori = (ori + 1) % 3;
      int t1 = dtri(S->nbr[index * 3 + ori]), t2 = dtri(S->nbr[index * 3 + (ori + 2) % 3]);
      if ((t1 < 0 || flipBy[t1] == index) && (t2 < 0 || flipBy[t2] == index)) win = 1;
    } else {
      ori -= 6;
      int pOpp = S->nbr[index * 3 + ori];
      int pOppTri = dtri(pOpp), pOppOri = dori(pOpp);
      int pOrg = S->tri[index * 3 + (ori + 1) % 3], pDest = S->tri[index * 3 + (ori + 2) % 3];
      int t1, t2;
      if ((S->ps[pOrg] & PS_REDUNDANT) &&
          (!(S->ps[pDest] & PS_REDUNDANT) || ((S->ps[pDest] & PS_REDUNDANT) && pOrg < pDest))) {
        t1 = S->nbr[index * 3 + (ori + 2) % 3];
        t2 = S->nbr[pOppTri * 3 + (pOppOri + 1) % 3];
      } else {
        t1 = S->nbr[index * 3 + (ori + 1) % 3];
        t2 = S->nbr[pOppTri * 3 + (pOppOri + 2) % 3];
      }
      t1 = dtri(t1);
      t2 = dtri(t2);
      if (flipBy[pOppTri] == index && flipBy[t1] == index && flipBy[t2] == index) win = 1;
    }
  }
  if (!win) ts_setflipori(&S->ts[index], 15);
}

/* kernelInitLinklist, refine.cu:1172-1278 */
static void init_linklist(St *S, int pos, int index, int *ll) {
  int ori = ts_flipori(S->ts[index]);
  if (ori < 3) {
    ll[4 * pos] = index;
    ll[4 * pos + 1] = dtri(S->nbr[index * 3 + (ori + 1) % 3]);
  } else if (ori < 6) {
    ori -= 3;
    ori = (ori + 1) % 3;
    ll[4 * pos] = index;
    ll[4 * pos + 1] = dtri(S->nbr[index * 3 + ori]);
    ll[4 * pos + 2] = dtri(S->nbr[index * 3 + (ori + 2) % 3]);
  } else {
    ori -= 6;
    int pOpp = S->nbr[index * 3 + ori];
    int pOppTri = dtri(pOpp), pOppOri = dori(pOpp);
    int min = MAXINT_REF;
    int p[3] = {S->tri[3 * pOppTri], S->tri[3 * pOppTri + 1], S->tri[3 * pOppTri + 2]};
    for (int i = 0; i < 3; i++)
      if ((S->ps[p[i]] & PS_REDUNDANT) && p[i] < min) min = p[i];
    int outward = (min == p[(pOppOri + 2) % 3]);
    int t1, t2;
    if (outward) {
      t1 = dtri(S->nbr[index * 3 + (ori + 2) % 3]);
      t2 = dtri(S->nbr[pOppTri * 3 + (pOppOri + 1) % 3]);
    } else {
      t1 = dtri(S->nbr[index * 3 + (ori + 1) % 3]);
      t2 = dtri(S->nbr[pOppTri * 3 + (pOppOri + 2) % 3]);
    }
    ll[4 * pos] = index;
    ll[4 * pos + 1] = pOppTri;
    ll[4 * pos + 2] = t1;
    ll[4 * pos + 3] = t2;
  }
}

static void set_tri(St *S, int a, int b, int c, int t, int ori) { /* setTriangle 1280 */
  S->tri[t * 3 + (ori + 1) % 3] = a;
  S->tri[t * 3 + (ori + 2) % 3] = b;
  S->tri[t * 3 + ori] = c;
}
static void set_link(int *sl, int nOrg, int nDest, int nApex, int li, int ori) { /* setNeighborlink 1287 */
  sl[li * 3 + ori] = nOrg;
  sl[li * 3 + (ori + 1) % 3] = nDest;
  sl[li * 3 + (ori + 2) % 3] = nApex;
}

/* kernelUpdatePhase1, refine.cu:1295-1552 */
static void phase1(St *S, int pos, int index, int *sl) {
  int ori = ts_flipori(S->ts[index]);
  if (ori < 3) {
    int pOpp = S->nbr[index * 3 + (ori + 1) % 3];
    int pOppTri = dtri(pOpp), pOppOri = dori(pOpp);
    int pOrg = S->tri[index * 3 + (ori + 1) % 3], pDest = S->tri[index * 3 + (ori + 2) % 3];
    int pApex = S->tri[index * 3 + ori];
    pOpp = S->tri[pOppTri * 3 + pOppOri];
    int nOrg = S->nbr[index * 3 + ori], nApex = S->nbr[index * 3 + (ori + 2) % 3];
    int npDest = S->nbr[pOppTri * 3 + (pOppOri + 1) % 3], npApex = S->nbr[pOppTri * 3 + (pOppOri + 2) % 3];
    set_tri(S, pOrg, pDest, pOpp, index, ori);
    set_tri(S, pApex, pOrg, pOpp, pOppTri, pOppOri);
    set_link(sl, nOrg + 3, MAXINT_REF, nApex + 3, 4 * pos, ori);
    set_link(sl, MAXINT_REF, npDest + 3, npApex + 3, 4 * pos + 1, pOppOri);
    int sOrg = S->t2s[3 * index + ori], sApex = S->t2s[3 * index + (ori + 2) % 3];
    int spDest = S->t2s[3 * pOppTri + (pOppOri + 1) % 3], spApex = S->t2s[3 * pOppTri + (pOppOri + 2) % 3];
    S->t2s[3 * index + ori] = sOrg;
    S->t2s[3 * index + (ori + 1) % 3] = spDest;
    S->t2s[3 * index + (ori + 2) % 3] = -1;
    S->t2s[3 * pOppTri + pOppOri] = sApex;
    S->t2s[3 * pOppTri + (pOppOri + 2) % 3] = spApex;
    S->t2s[3 * pOppTri + (pOppOri + 1) % 3] = -1;
    if (sOrg != -1) s2t_set(S, sOrg, (index << 2) | ori, wkey(pos, 0));
    if (spDest != -1) s2t_set(S, spDest, (index << 2) | ((ori + 1) % 3), wkey(pos, 1));
    if (sApex != -1) s2t_set(S, sApex, (pOppTri << 2) | pOppOri, wkey(pos, 2));
    if (spApex != -1) s2t_set(S, spApex, (pOppTri << 2) | ((pOppOri + 2) % 3), wkey(pos, 3));
    ts_set(&S->ts[index], TS_CHECK, 1);
    ts_set(&S->ts[pOppTri], TS_CHECK, 1);
  } else if (ori < 6) {
    ori -= 3;
    ori = (ori + 1) % 3;
    int t1 = S->nbr[index * 3 + ori], t2 = S->nbr[index * 3 + (ori + 2) % 3];
    int t1_ori = dori(t1), t2_ori = dori(t2);
    t1 = dtri(t1);
    t2 = dtri(t2);
    int pOrg = S->tri[index * 3 + (ori + 1) % 3], pDest = S->tri[index * 3 + (ori + 2) % 3];
    int pApex = S->tri[index * 3 + ori];
    S->ps[pOrg] |= PS_DELETED;
    pOrg = S->tri[t1 * 3 + t1_ori];
    int nOrg = S->nbr[t1 * 3 + (t1_ori + 2) % 3], nDest = S->nbr[index * 3 + (ori + 1) % 3];
    int nApex = S->nbr[t2 * 3 + (t2_ori + 1) % 3];
    set_tri(S, pOrg, pDest, pApex, index, ori);
    set_link(sl, nOrg + 3, nDest + 3, nApex + 3, 4 * pos, ori);
    sl[(4 * pos + 1) * 3 + (t1_ori + 2) % 3] = nOrg + 3;
    sl[(4 * pos + 2) * 3 + (t2_ori + 1) % 3] = nApex + 3;
    int sOrg = S->t2s[3 * index + (ori + 1) % 3], sApex = S->t2s[3 * t1 + (t1_ori + 2) % 3];
    int sDest = S->t2s[3 * t2 + (t2_ori + 1) % 3];
    S->t2s[3 * index + (ori + 1) % 3] = sOrg;
    S->t2s[3 * index + ori] = sApex;
    S->t2s[3 * index + (ori + 2) % 3] = sDest;
    if (sOrg != -1) s2t_set(S, sOrg, (index << 2) | ((ori + 1) % 3), wkey(pos, 4));
    if (sApex != -1) s2t_set(S, sApex, (index << 2) | ori, wkey(pos, 5));
    if (sDest != -1) s2t_set(S, sDest, (index << 2) | ((ori + 2) % 3), wkey(pos, 6));
    ts_set(&S->ts[index], TS_CHECK, 1);
    ts_set(&S->ts[t1], TS_NOTNULL, 0);
    ts_set(&S->ts[t2], TS_NOTNULL, 0);
  } else {
    ori -= 6;
    int pOpp = S->nbr[index * 3 + ori];
    int pOppTri = dtri(pOpp), pOppOri = dori(pOpp);
    int pOrg = S->tri[index * 3 + (ori + 1) % 3], pDest = S->tri[index * 3 + (ori + 2) % 3];
    int pApex = S->tri[index * 3 + ori];
    pOpp = S->tri[pOppTri * 3 + pOppOri];
    int t1, t2, t1_ori, t2_ori;
    int outw = (S->ps[pOrg] & PS_REDUNDANT) &&
               (!(S->ps[pDest] & PS_REDUNDANT) || ((S->ps[pDest] & PS_REDUNDANT) && pOrg < pDest));
    if (outw) {
      t1 = S->nbr[index * 3 + (ori + 2) % 3];
      t2 = S->nbr[pOppTri * 3 + (pOppOri + 1) % 3];
    } else {
      t1 = S->nbr[index * 3 + (ori + 1) % 3];
      t2 = S->nbr[pOppTri * 3 + (pOppOri + 2) % 3];
    }
    t1_ori = dori(t1);
    t2_ori = dori(t2);
    t1 = dtri(t1);
    t2 = dtri(t2);
    int nOpp = S->tri[3 * t1 + t1_ori];
    int sOrg, sDest, sApex, snOrg, snDest, snApex;
    if (outw) {
      S->ps[pOrg] |= PS_DELETED;
      int nOrg = S->nbr[pOppTri * 3 + (pOppOri + 2) % 3], nDest = S->nbr[index * 3 + (ori + 1) % 3];
      int npDest = S->nbr[t1 * 3 + (t1_ori + 1) % 3], npApex = S->nbr[t2 * 3 + (t2_ori + 2) % 3];
      set_tri(S, pOpp, pDest, pApex, index, ori);
      set_tri(S, pOpp, pApex, nOpp, t1, t1_ori);
      set_link(sl, nOrg + 3, nDest + 3, MAXINT_REF, 4 * pos, ori);
      set_link(sl, MAXINT_REF, npDest + 3, npApex + 3, 4 * pos + 2, t1_ori);
      sl[(4 * pos + 1) * 3 + (pOppOri + 2) % 3] = nOrg + 3;
      sl[(4 * pos + 3) * 3 + (t2_ori + 2) % 3] = npApex + 3;
      sOrg = S->t2s[3 * pOppTri + (pOppOri + 2) % 3];
      sDest = S->t2s[3 * index + (ori + 1) % 3];
      sApex = S->t2s[3 * index + (ori + 2) % 3];
      snOrg = S->t2s[3 * t1 + t1_ori];
      snDest = S->t2s[3 * t1 + (t1_ori + 1) % 3];
      snApex = S->t2s[3 * t2 + (t2_ori + 2) % 3];
    } else {
      S->ps[pDest] |= PS_DELETED;
      int nOrg = S->nbr[pOppTri * 3 + (pOppOri + 1) % 3], nApex = S->nbr[index * 3 + (ori + 2) % 3];
      int npDest = S->nbr[t2 * 3 + (t2_ori + 1) % 3], npApex = S->nbr[t1 * 3 + (t1_ori + 2) % 3];
      set_tri(S, pOrg, pOpp, pApex, index, ori);
      set_tri(S, pApex, pOpp, nOpp, t1, t1_ori);
      set_link(sl, nOrg + 3, MAXINT_REF, nApex + 3, 4 * pos, ori);
      set_link(sl, MAXINT_REF, npDest + 3, npApex + 3, 4 * pos + 2, t1_ori);
      sl[(4 * pos + 1) * 3 + (pOppOri + 1) % 3] = nOrg + 3;
      sl[(4 * pos + 3) * 3 + (t2_ori + 1) % 3] = npDest + 3;
      sOrg = S->t2s[3 * pOppTri + (pOppOri + 1) % 3];
      sDest = S->t2s[3 * index + (ori + 1) % 3];
      sApex = S->t2s[3 * index + (ori + 2) % 3];
      snOrg = S->t2s[3 * t1 + t1_ori];
      snDest = S->t2s[3 * t2 + (t2_ori + 1) % 3];
      snApex = S->t2s[3 * t1 + (t1_ori + 2) % 3];
    }
    S->t2s[3 * index + ori] = sOrg;
    S->t2s[3 * index + (ori + 1) % 3] = sDest;
    S->t2s[3 * index + (ori + 2) % 3] = sApex;
    S->t2s[3 * t1 + t1_ori] = snOrg;
    S->t2s[3 * t1 + (t1_ori + 1) % 3] = snDest;
    S->t2s[3 * t1 + (t1_ori + 2) % 3] = snApex;
    if (sOrg != -1) s2t_set(S, sOrg, (index << 2) | ori, wkey(pos, 7));
    if (sDest != -1) s2t_set(S, sDest, (index << 2) | ((ori + 1) % 3), wkey(pos, 8));
    if (sApex != -1) s2t_set(S, sApex, (index << 2) | ((ori + 2) % 3), wkey(pos, 9));
    if (snOrg != -1) s2t_set(S, snOrg, (t1 << 2) | t1_ori, wkey(pos, 10));
    if (snDest != -1) s2t_set(S, snDest, (t1 << 2) | ((t1_ori + 1) % 3), wkey(pos, 11));
    if (snApex != -1) s2t_set(S, snApex, (t1 << 2) | ((t1_ori + 2) % 3), wkey(pos, 12));
    ts_set(&S->ts[index], TS_CHECK, 1);
    ts_set(&S->ts[t1], TS_CHECK, 1);
    ts_set(&S->ts[pOppTri], TS_NOTNULL, 0);
    ts_set(&S->ts[t2], TS_NOTNULL, 0);
  }
}

/* updateNeighborlink, refine.cu:1554-1596 */
static void update_link(const int *ll, int *sl, int wIndex, int otri, int neighbor, int nw) {
  int low = 0, high = nw - 1, listIndex = -1, found = 0;
  int triIndex = dtri(otri), triOri = dori(otri);
  while (high >= low) {
    int middle = (low + high) / 2;
    int windex = ll[4 * middle];
    if (windex == wIndex) {
      for (int i = 0; i < 4; i++)
        if (ll[4 * middle + i] == triIndex) {
          listIndex = 4 * middle + i;
          found = 1;
          break;
        }
      if (found) break;
    } else if (windex < wIndex)
      low = middle + 1;
    else
      high = middle - 1;
  }
  if (listIndex >= 0) sl[listIndex * 3 + triOri] = -neighbor;
}
static void p2_try(St *S, const int *ll, int *sl, int nlink, int neighbor, int nw) {
  int tempIndex = dtri(nlink);
  if (tempIndex != -1) {
    int w = S->tmark[tempIndex];
    if (w != MAXINT_REF && w >= 0 && ts_flipori(S->ts[w]) != 15) update_link(ll, sl, w, nlink, neighbor, nw);
  }
}

/* kernelUpdatePhase2, refine.cu:1598-1871 */
static void phase2(St *S, int index, const int *ll, int *sl, int nw) {
  int ori = ts_flipori(S->ts[index]);
  if (ori < 3) {
    int pOpp = S->nbr[index * 3 + (ori + 1) % 3];
    int pOppTri = dtri(pOpp), pOppOri = dori(pOpp);
    int nOrg = S->nbr[index * 3 + ori], nApex = S->nbr[index * 3 + (ori + 2) % 3];
    int npDest = S->nbr[pOppTri * 3 + (pOppOri + 1) % 3], npApex = S->nbr[pOppTri * 3 + (pOppOri + 2) % 3];
    p2_try(S, ll, sl, nOrg, etri(index, ori), nw);
    p2_try(S, ll, sl, nApex, etri(pOppTri, pOppOri), nw);
    p2_try(S, ll, sl, npDest, etri(index, (ori + 1) % 3), nw);
    p2_try(S, ll, sl, npApex, etri(pOppTri, (pOppOri + 2) % 3), nw);
  } else if (ori < 6) {
    ori -= 3;
    ori = (ori + 1) % 3;
    int t1 = S->nbr[index * 3 + ori], t2 = S->nbr[index * 3 + (ori + 2) % 3];
    int t1_ori = dori(t1), t2_ori = dori(t2);
    t1 = dtri(t1);
    t2 = dtri(t2);
    int nOrg = S->nbr[t1 * 3 + (t1_ori + 2) % 3], nDest = S->nbr[index * 3 + (ori + 1) % 3];
    int nApex = S->nbr[t2 * 3 + (t2_ori + 1) % 3];
    p2_try(S, ll, sl, nOrg, etri(index, ori), nw);
    p2_try(S, ll, sl, nDest, etri(index, (ori + 1) % 3), nw);
    p2_try(S, ll, sl, nApex, etri(index, (ori + 2) % 3), nw);
  } else {
    ori -= 6;
    int pOpp = S->nbr[index * 3 + ori];
    int pOppTri = dtri(pOpp), pOppOri = dori(pOpp);
    int min = MAXINT_REF;
    int p[3] = {S->tri[3 * pOppTri], S->tri[3 * pOppTri + 1], S->tri[3 * pOppTri + 2]};
    for (int i = 0; i < 3; i++)
      if ((S->ps[p[i]] & PS_REDUNDANT) && p[i] < min) min = p[i];
    int outward = (min == p[(pOppOri + 2) % 3]);
    if (outward) {
      int t1 = S->nbr[index * 3 + (ori + 2) % 3], t2 = S->nbr[pOppTri * 3 + (pOppOri + 1) % 3];
      int t1_ori = dori(t1), t2_ori = dori(t2);
      t1 = dtri(t1);
      t2 = dtri(t2);
      int nOrg = S->nbr[3 * pOppTri + (pOppOri + 2) % 3], nDest = S->nbr[3 * index + (ori + 1) % 3];
      int npDest = S->nbr[3 * t1 + (t1_ori + 1) % 3], npApex = S->nbr[3 * t2 + (t2_ori + 2) % 3];
      p2_try(S, ll, sl, nOrg, etri(index, ori), nw);
      p2_try(S, ll, sl, nDest, etri(index, (ori + 1) % 3), nw);
      p2_try(S, ll, sl, npDest, etri(t1, (t1_ori + 1) % 3), nw);
      p2_try(S, ll, sl, npApex, etri(t1, (t1_ori + 2) % 3), nw);
    } else {
      int t1 = S->nbr[index * 3 + (ori + 1) % 3], t2 = S->nbr[pOppTri * 3 + (pOppOri + 2) % 3];
      int t1_ori = dori(t1), t2_ori = dori(t2);
      t1 = dtri(t1);
      t2 = dtri(t2);
      int nOrg = S->nbr[3 * pOppTri + (pOppOri + 1) % 3], nApex = S->nbr[3 * index + (ori + 2) % 3];
      int npDest = S->nbr[3 * t2 + (t2_ori + 1) % 3], npApex = S->nbr[3 * t1 + (t1_ori + 2) % 3];
      p2_try(S, ll, sl, nOrg, etri(index, ori), nw);
      p2_try(S, ll, sl, nApex, etri(index, (ori + 2) % 3), nw);
      p2_try(S, ll, sl, npDest, etri(t1, (t1_ori + 1) % 3), nw);
      p2_try(S, ll, sl, npApex, etri(t1, (t1_ori + 2) % 3), nw);
    }
  }
}

/* resetEncseg, refine.cu:1879-1922 */
static void reset_encseg(St *S, int s, int otri0, int otri1) {
  S->enc.a[s] = -1;
  if (otri0 != -1) {
    int t = dtri(otri0), o = dori(otri0);
    P2 vo = S->pts[S->tri[3 * t + (o + 1) % 3]], vd = S->pts[S->tri[3 * t + (o + 2) % 3]];
    P2 va = S->pts[S->tri[3 * t + o]];
    if (encroached(vo, vd, va, S->gc2, S->mode)) S->enc.a[s] = 0;
  }
  if (otri1 != -1) {
    int t = dtri(otri1), o = dori(otri1);
    P2 vo = S->pts[S->tri[3 * t + (o + 1) % 3]], vd = S->pts[S->tri[3 * t + (o + 2) % 3]];
    P2 va = S->pts[S->tri[3 * t + o]];
    if (encroached(vo, vd, va, S->gc2, S->mode)) S->enc.a[s] = 0;
  }
}
static void upd_nl(St *S, int t, int v) { /* updateNeighborlist 1873 */
  if (t >= 0) S->nbr[dtri(t) * 3 + dori(t)] = v;
}
static int unlink_slot(St *S, int v, int newlink) {
  /* v > 0: the neighbour did not update me; update him (refine.cu:1974-1992) */
  if (v > 0) {
    v = -(v - 3);
    upd_nl(S, -v, newlink);
  }
  return v;
}

/* kernelUpdatePhase3, refine.cu:1924-2296 */
static void phase3(St *S, int pos, int index, const int *sl) {
  int ori = ts_flipori(S->ts[index]);
  ts_setflipori(&S->ts[index], 15);
  if (ori < 3) {
    int pOpp = S->nbr[index * 3 + (ori + 1) % 3];
    int pOppTri = dtri(pOpp), pOppOri = dori(pOpp);
    int nOrg = sl[4 * pos * 3 + ori], nApex = sl[4 * pos * 3 + (ori + 2) % 3];
    int npDest = sl[(4 * pos + 1) * 3 + (pOppOri + 1) % 3], npApex = sl[(4 * pos + 1) * 3 + (pOppOri + 2) % 3];
    nOrg = unlink_slot(S, nOrg, etri(index, ori));
    nApex = unlink_slot(S, nApex, etri(pOppTri, pOppOri));
    npDest = unlink_slot(S, npDest, etri(index, (ori + 1) % 3));
    npApex = unlink_slot(S, npApex, etri(pOppTri, (pOppOri + 2) % 3));
    S->nbr[index * 3 + ori] = -nOrg;
    S->nbr[index * 3 + (ori + 1) % 3] = -npDest;
    S->nbr[index * 3 + (ori + 2) % 3] = etri(pOppTri, (pOppOri + 1) % 3);
    S->nbr[pOppTri * 3 + pOppOri] = -nApex;
    S->nbr[pOppTri * 3 + (pOppOri + 1) % 3] = etri(index, (ori + 2) % 3);
    S->nbr[pOppTri * 3 + (pOppOri + 2) % 3] = -npApex;
    int sOrg = S->t2s[3 * index + ori], sDest = S->t2s[3 * index + (ori + 1) % 3];
    int spOrg = S->t2s[3 * pOppTri + pOppOri], spApex = S->t2s[3 * pOppTri + (pOppOri + 2) % 3];
    if (sOrg != -1) reset_encseg(S, sOrg, (index << 2) | ori, -nOrg);
    if (sDest != -1) reset_encseg(S, sDest, (index << 2) | ((ori + 1) % 3), -npDest);
    if (spOrg != -1) reset_encseg(S, spOrg, (pOppTri << 2) | pOppOri, -nApex);
    if (spApex != -1) reset_encseg(S, spApex, (pOppTri << 2) | ((pOppOri + 2) % 3), -npApex);
    ts_set(&S->ts[pOppTri], TS_FLIP, 1);
  } else if (ori < 6) {
    ori -= 3;
    ori = (ori + 1) % 3;
    int t1 = S->nbr[index * 3 + ori], t2 = S->nbr[index * 3 + (ori + 2) % 3];
    int t1_ori = dori(t1), t2_ori = dori(t2);
    t1 = dtri(t1);
    t2 = dtri(t2);
    int nOrg = sl[(4 * pos + 1) * 3 + (t1_ori + 2) % 3], nDest = sl[4 * pos * 3 + (ori + 1) % 3];
    int nApex = sl[(4 * pos + 2) * 3 + (t2_ori + 1) % 3];
    nOrg = unlink_slot(S, nOrg, etri(index, ori));
    nDest = unlink_slot(S, nDest, etri(index, (ori + 1) % 3));
    nApex = unlink_slot(S, nApex, etri(index, (ori + 2) % 3));
    S->nbr[index * 3 + ori] = -nOrg;
    S->nbr[index * 3 + (ori + 1) % 3] = -nDest;
    S->nbr[index * 3 + (ori + 2) % 3] = -nApex;
    int sOrg = S->t2s[3 * index + ori], sDest = S->t2s[3 * index + (ori + 1) % 3];
    int sApex = S->t2s[3 * index + (ori + 2) % 3];
    if (sOrg != -1) reset_encseg(S, sOrg, (index << 2) | ori, -nOrg);
    if (sDest != -1) reset_encseg(S, sDest, (index << 2) | ((ori + 1) % 3), -nDest);
    if (sApex != -1) reset_encseg(S, sApex, (index << 2) | ((ori + 2) % 3), -nApex);
    ts_set(&S->ts[t1], TS_FLIP, 0);
    ts_set(&S->ts[t2], TS_FLIP, 0);
  } else {
    ori -= 6;
    int pOpp = S->nbr[index * 3 + ori];
    int pOppTri = dtri(pOpp), pOppOri = dori(pOpp);
    int min = MAXINT_REF;
    int p[3] = {S->tri[3 * pOppTri], S->tri[3 * pOppTri + 1], S->tri[3 * pOppTri + 2]};
    for (int i = 0; i < 3; i++)
      if ((S->ps[p[i]] & PS_REDUNDANT) && p[i] < min) min = p[i];
    int outward = (min == p[(pOppOri + 2) % 3]);
    int t1, t2, t1_ori, t2_ori;
    if (outward) {
      t1 = S->nbr[index * 3 + (ori + 2) % 3];
      t2 = S->nbr[pOppTri * 3 + (pOppOri + 1) % 3];
      t1_ori = dori(t1);
      t2_ori = dori(t2);
      t1 = dtri(t1);
      t2 = dtri(t2);
      int nOrg = sl[(4 * pos + 1) * 3 + (pOppOri + 2) % 3], nDest = sl[4 * pos * 3 + (ori + 1) % 3];
      int npDest = sl[(4 * pos + 2) * 3 + (t1_ori + 1) % 3], npApex = sl[(4 * pos + 3) * 3 + (t2_ori + 2) % 3];
      nOrg = unlink_slot(S, nOrg, etri(index, ori));
      nDest = unlink_slot(S, nDest, etri(index, (ori + 1) % 3));
      npDest = unlink_slot(S, npDest, etri(t1, (t1_ori + 1) % 3));
      npApex = unlink_slot(S, npApex, etri(t1, (t1_ori + 2) % 3));
      S->nbr[index * 3 + ori] = -nOrg;
      S->nbr[index * 3 + (ori + 1) % 3] = -nDest;
      S->nbr[t1 * 3 + (t1_ori + 1) % 3] = -npDest;
      S->nbr[t1 * 3 + (t1_ori + 2) % 3] = -npApex;
      int sOrg = S->t2s[3 * index + ori], sDest = S->t2s[3 * index + (ori + 1) % 3];
      int spDest = S->t2s[3 * t1 + (t1_ori + 1) % 3], spApex = S->t2s[3 * t1 + (t1_ori + 2) % 3];
      if (sOrg != -1) reset_encseg(S, sOrg, (index << 2) | ori, -nOrg);
      if (sDest != -1) reset_encseg(S, sDest, (index << 2) | ((ori + 1) % 3), -nDest);
      if (spDest != -1) reset_encseg(S, spDest, (t1 << 2) | ((t1_ori + 1) % 3), -npDest);
      if (spApex != -1) reset_encseg(S, spApex, (t1 << 2) | ((t1_ori + 2) % 3), -npApex);
    } else {
      t1 = S->nbr[index * 3 + (ori + 1) % 3];
      t2 = S->nbr[pOppTri * 3 + (pOppOri + 2) % 3];
      t1_ori = dori(t1);
      t2_ori = dori(t2);
      t1 = dtri(t1);
      t2 = dtri(t2);
      int nOrg = sl[(4 * pos + 1) * 3 + (pOppOri + 1) % 3], nApex = sl[4 * pos * 3 + (ori + 2) % 3];
      int npDest = sl[(4 * pos + 3) * 3 + (t2_ori + 1) % 3], npApex = sl[(4 * pos + 2) * 3 + (t1_ori + 2) % 3];
      nOrg = unlink_slot(S, nOrg, etri(index, ori));
      nApex = unlink_slot(S, nApex, etri(index, (ori + 2) % 3));
      npDest = unlink_slot(S, npDest, etri(t1, (t1_ori + 1) % 3));
      npApex = unlink_slot(S, npApex, etri(t1, (t1_ori + 2) % 3));
      S->nbr[index * 3 + ori] = -nOrg;
      S->nbr[index * 3 + (ori + 2) % 3] = -nApex;
      S->nbr[t1 * 3 + (t1_ori + 1) % 3] = -npDest;
      S->nbr[t1 * 3 + (t1_ori + 2) % 3] = -npApex;
      int sOrg = S->t2s[3 * index + ori], sApex = S->t2s[3 * index + (ori + 2) % 3];
      int spDest = S->t2s[3 * t1 + (t1_ori + 1) % 3], spApex = S->t2s[3 * t1 + (t1_ori + 2) % 3];
      if (sOrg != -1) reset_encseg(S, sOrg, (index << 2) | ori, -nOrg);
      if (sApex != -1) reset_encseg(S, sApex, (index << 2) | ((ori + 2) % 3), -nApex);
      if (spDest != -1) reset_encseg(S, spDest, (t1 << 2) | ((t1_ori + 1) % 3), -npDest);
      if (spApex != -1) reset_encseg(S, spApex, (t1 << 2) | ((t1_ori + 2) % 3), -npApex);
    }
    ts_set(&S->ts[t1], TS_FLIP, 1);
    ts_set(&S->ts[pOppTri], TS_FLIP, 0);
    ts_set(&S->ts[t2], TS_FLIP, 0);
  }
}

/* kernelMarkReduntantSteiner, refine.cu:2298-2326 */
static void mark_redundant_steiner(St *S, int index) {
  int otri = negate_ref(S->tmark[index]);
  int triIndex = dtri(otri), triOri = dori(otri);
  if (triIndex != index) ts_set(&S->ts[index], TS_FLIP, 1);
  int pindex = S->tri[3 * triIndex + (triOri + 1) % 3];
  S->ps[pindex] |= PS_REDUNDANT;
  mark_fan(S, triIndex, triOri);
}

/* flipFlop, refine.cu:2328-2490 */
/* ---------------- step trace (debugging aid of the test infrastructure) ----------------
 * When enabled, one line per flip step with FNV-1a digests of the mesh arrays
 * as kernelCheckFlipping (refine.cu:778) sees them at launch: the same line
 * can be produced from the reference by interposing on its kernel launches,
 * which finds the first step at which two runs part. */
static FILE *g_trace;
static long g_trace_seq, g_dump_step = -1;
static char g_dump_path[512];
void gqm_oracle_trace(const char *path) {
  if (g_trace) fclose(g_trace);
  g_trace = path ? fopen(path, "w") : NULL;
  g_trace_seq = 0;
}
/* Also write the full arrays of flip step `step` (same layout as the trace's
 * digests, after a 4-int header) to `path`. */
void gqm_oracle_trace_dump(long step, const char *path) {
  g_dump_step = path ? step : -1;
  if (path) snprintf(g_dump_path, sizeof g_dump_path, "%s", path);
}
static unsigned long long fnv64(const void *p, size_t n) {
  const unsigned char *b = (const unsigned char *)p;
  unsigned long long h = 1469598103934665603ULL;
  for (size_t i = 0; i < n; ++i) {
    h ^= b[i];
    h *= 1099511628211ULL;
  }
  return h;
}
static int cmp_tri3(const void *a, const void *b) {
  const int *x = (const int *)a, *y = (const int *)b;
  for (int i = 0; i < 3; ++i)
    if (x[i] != y[i]) return x[i] < y[i] ? -1 : 1;
  return 0;
}
/* digest of the live triangles as a set: each rotated to start at its
 * smallest vertex (orientation kept), sorted */
static unsigned long long mesh_digest(const int *tri, const unsigned char *ts, int ntri) {
  int *c = (int *)malloc(sizeof(int) * 3 * ((size_t)ntri + 1));
  long m = 0;
  for (int t = 0; t < ntri; ++t) {
    if (!(ts[t] & TS_NOTNULL)) continue;
    int a = tri[3 * t], b = tri[3 * t + 1], d = tri[3 * t + 2];
    int k = (a <= b && a <= d) ? 0 : (b <= d ? 1 : 2);
    int v[3] = {a, b, d};
    for (int i = 0; i < 3; ++i) c[3 * m + i] = v[(k + i) % 3];
    m++;
  }
  qsort(c, (size_t)m, sizeof(int) * 3, cmp_tri3);
  unsigned long long h = fnv64(c, sizeof(int) * 3 * (size_t)m);
  free(c);
  return h;
}
static void trace_flip_step(St *S, int ntri, const IV *act) {
  if (!g_trace) return;
  int np = 0;
  for (long i = 0; i < 3L * ntri; ++i)
    if (S->tri[i] + 1 > np) np = S->tri[i] + 1;
  fprintf(g_trace,
          "F %ld nt=%d nact=%ld tri=%016llx nbr=%016llx t2s=%016llx ts=%016llx act=%016llx np=%d pts=%016llx "
          "mesh=%016llx\n",
          g_trace_seq++, ntri, act->n, fnv64(S->tri, sizeof(int) * 3L * ntri), fnv64(S->nbr, sizeof(int) * 3L * ntri),
          fnv64(S->t2s, sizeof(int) * 3L * ntri), fnv64(S->ts, (size_t)ntri), fnv64(act->a, sizeof(int) * act->n), np,
          fnv64(S->pts, sizeof(P2) * (size_t)np), mesh_digest(S->tri, S->ts, ntri));
  fflush(g_trace);
  if (g_trace_seq - 1 == g_dump_step) {
    FILE *d = fopen(g_dump_path, "wb");
    if (d) {
      int hdr[4] = {(int)(g_trace_seq - 1), ntri, (int)act->n, np};
      fwrite(hdr, 4, 4, d);
      fwrite(S->tri, 4, 3L * ntri, d);
      fwrite(S->nbr, 4, 3L * ntri, d);
      fwrite(S->t2s, 4, 3L * ntri, d);
      fwrite(S->ts, 1, (size_t)ntri, d);
      fwrite(act->a, 4, (size_t)act->n, d);
      fwrite(S->pts, sizeof(P2), (size_t)np, d);
      fclose(d);
    }
  }
}

static void flip_flop(St *S, int ntri) {
  IV *act = &S->l3, *ll = &S->l4, *sl = &S->l5;
  unsigned char *flip0 = (unsigned char *)malloc((size_t)ntri + 1);
  long long steps = 0;
  for (;;) {
    act->n = 0;
    for (int t = 0; t < ntri; ++t)
      if (!ts_null(S->ts[t]) && (S->ts[t] & TS_FLIP)) iv_push(act, t);
    if (act->n == 0) break;
    if (S->max_rounds && ++steps > 64 * S->max_rounds) {
      S->err = -2;
      break;
    }
    S->flip_steps++;
    for (int t = 0; t < ntri; ++t) S->tmark[t] = MAXINT_REF;
    for (int t = 0; t < ntri; ++t) ts_setflipori(&S->ts[t], 15);
    for (int t = 0; t < ntri; ++t) flip0[t] = (S->ts[t] & TS_FLIP) ? 1 : 0;
    trace_flip_step(S, ntri, act);
    for (long k = 0; k < act->n; ++k) check_flipping(S, act->a[k], flip0);
    for (long k = 0; k < act->n; ++k) mark_flip_winner(S, act->a[k]);
    /* winners: not null and flipOri != 15, ascending */
    IV win = {0, 0, 0};
    for (int t = 0; t < ntri; ++t)
      if (!ts_null(S->ts[t]) && ts_flipori(S->ts[t]) != 15) iv_push(&win, t);
    int nw = (int)win.n;
    iv_resize(ll, 0, 0);
    iv_resize(ll, 4L * nw, -1);
    iv_resize(sl, 12L * nw, 0);
    for (int k = 0; k < nw; ++k) init_linklist(S, k, win.a[k], ll->a);
    s2t_begin(S);
    for (int k = 0; k < nw; ++k) phase1(S, k, win.a[k], sl->a);
    for (int k = 0; k < nw; ++k) phase2(S, win.a[k], ll->a, sl->a, nw);
    for (int k = 0; k < nw; ++k) phase3(S, k, win.a[k], sl->a);
    free(win.a);
    IV neg = {0, 0, 0};
    for (int t = 0; t < ntri; ++t)
      if (S->tmark[t] < 0) iv_push(&neg, t);
    for (long k = 0; k < neg.n; ++k) mark_redundant_steiner(S, neg.a[k]);
    free(neg.a);
    if (S->err) break;
  }
  free(flip0);
}

/* ---------------- encroached subsegments (refine.cu:2492-3778) ---------------- */
/* kernelMarkReduantPoints thread body, refine.cu:604-677 */
static void mark_redundant_points(St *S, int pos, int *delmarker, const int *dellist) {
  delmarker[pos] = -1;
  int sindex = dellist[pos];
  int otri = S->s2t.a[sindex];
  int triIndex = dtri(otri), triOri = dori(otri);
  int pOrg = S->tri[3 * triIndex + (triOri + 1) % 3], pDest = S->tri[3 * triIndex + (triOri + 2) % 3];
  int pApex = S->tri[3 * triIndex + triOri];
  P2 vOrg = S->pts[pOrg], vDest = S->pts[pDest], vApex = S->pts[pApex];
  if ((S->ps[pApex] & PS_STEINER) && !(S->ps[pApex] & PS_SEGSPLIT) &&
      ((vOrg.x - vApex.x) * (vDest.x - vApex.x) + (vOrg.y - vApex.y) * (vDest.y - vApex.y) < 0.0)) {
    S->ps[pApex] |= PS_REDUNDANT;
    mark_fan(S, triIndex, (triOri + 2) % 3);
    delmarker[pos] = sindex;
  }
  otri = S->nbr[3 * triIndex + triOri];
  if (otri != -1) {
    triIndex = dtri(otri);
    triOri = dori(otri);
    pApex = S->tri[3 * triIndex + triOri];
    vApex = S->pts[pApex];
    if ((S->ps[pApex] & PS_STEINER) && !(S->ps[pApex] & PS_SEGSPLIT) &&
        ((vOrg.x - vApex.x) * (vDest.x - vApex.x) + (vOrg.y - vApex.y) * (vDest.y - vApex.y) < 0.0)) {
      S->ps[pApex] |= PS_REDUNDANT;
      mark_fan(S, triIndex, (triOri + 2) % 3);
      delmarker[pos] = sindex;
    }
  }
}

static void insert_tri(St *S, int v0, int v1, int v2, int t, int nA, int nO, int nD) { /* insertTriangle 2581 */
  if (t >= 0) {
    S->tri[t * 3] = v0;
    S->tri[t * 3 + 1] = v1;
    S->tri[t * 3 + 2] = v2;
    S->nbr[t * 3] = nA;
    S->nbr[t * 3 + 1] = nO;
    S->nbr[t * 3 + 2] = nD;
  }
}

/* kernelInsertMidPoints, refine.cu:2594-2927 (debug printing omitted) */
static void insert_midpoint(St *S, int pos, int tindex, int *imarker, int nsub, int otri) {
  int sindex = imarker[tindex];
  int tri[4], p[3], neighbor[3], seg[3], triOri[2];
  int acuteorg = 0, acutedest = 0;
  tri[0] = dtri(otri);
  triOri[0] = dori(otri);
  if (S->tmark[tri[0]] != sindex) return;
  if (S->t2s[3 * tri[0] + (triOri[0] + 1) % 3] != -1) acutedest = 1;
  if (S->t2s[3 * tri[0] + (triOri[0] + 2) % 3] != -1) acuteorg = 1;
  otri = S->nbr[3 * tri[0] + triOri[0]];
  tri[2] = dtri(otri);
  triOri[1] = dori(otri);
  if (tri[2] != -1 && S->tmark[tri[2]] != sindex) return;
  if (tri[2] != -1) {
    if (S->t2s[3 * tri[2] + (triOri[1] + 1) % 3] != -1) acuteorg = 1;
    if (S->t2s[3 * tri[2] + (triOri[1] + 2) % 3] != -1) acutedest = 1;
  }
  int newp = new_point_slot(S, tindex);
  int nt1 = new_tri_slot(S, 2 * tindex), nt2 = new_tri_slot(S, 2 * tindex + 1);
  S->ps[newp] = PS_STEINER | PS_NEW | PS_SEGSPLIT;
  tri[1] = nt1;
  tri[3] = nt2;
  S->ts[tri[1]] = 0;
  S->ts[tri[3]] = 0;
  S->enc.a[sindex] = -1;
  S->enc.a[nsub + tindex] = -1;
  ts_set(&S->ts[tri[0]], TS_CHECK, 1);
  ts_set(&S->ts[tri[0]], TS_FLIP, 1);
  ts_setflipori(&S->ts[tri[0]], 0);
  ts_set(&S->ts[tri[1]], TS_NOTNULL, 1);
  ts_set(&S->ts[tri[1]], TS_CHECK, 1);
  ts_set(&S->ts[tri[1]], TS_FLIP, 1);
  ts_setflipori(&S->ts[tri[1]], 0);
  for (int i = 0; i < 3; i++) p[i] = S->tri[tri[0] * 3 + (triOri[0] + i + 1) % 3];
  P2 a = S->pts[p[0]], b = S->pts[p[1]];
  double segmentlength = sqrt(madd(a.x - b.x, a.x - b.x, (a.y - b.y) * (a.y - b.y)));
  double split = 0.5;
  if (acuteorg || acutedest) {
    double npt = 1.0;
    while (segmentlength > 3.0 * npt) npt *= 2.0;
    while (segmentlength < 1.5 * npt) npt *= 0.5;
    split = npt / segmentlength;
    if (acutedest) split = 1.0 - split;
  }
  S->pts[newp].x = madd(b.x - a.x, split, a.x);
  S->pts[newp].y = madd(b.y - a.y, split, a.y);
  double multiplier = orient_ref(a, b, S->pts[newp]);
  double divisor = madd(a.x - b.x, a.x - b.x, (a.y - b.y) * (a.y - b.y));
  if ((multiplier != 0.0) && (divisor != 0.0)) {
    multiplier = multiplier / divisor;
    if (multiplier == multiplier) {
      S->pts[newp].x = madd(multiplier, b.y - a.y, S->pts[newp].x);
      S->pts[newp].y = madd(multiplier, a.x - b.x, S->pts[newp].y);
    }
  }
  for (int i = 0; i < 3; i++) seg[i] = S->t2s[3 * tri[0] + (triOri[0] + i) % 3];
  S->t2s[3 * tri[0]] = seg[2];
  S->t2s[3 * tri[0] + 1] = seg[0];
  S->t2s[3 * tri[0] + 2] = -1;
  S->t2s[3 * tri[1]] = seg[1];
  S->t2s[3 * tri[1] + 1] = -1;
  S->t2s[3 * tri[1] + 2] = nsub + tindex;
  s2t_set(S, seg[0], (tri[0] << 2) | 1, wkey(pos, 0));
  s2t_set(S, nsub + tindex, (tri[1] << 2) | 2, wkey(pos, 1));
  S->s2seg.a[nsub + tindex] = S->s2seg.a[seg[0]];
  if (seg[1] != -1) s2t_set(S, seg[1], tri[1] << 2 | 0, wkey(pos, 2));
  if (seg[2] != -1) s2t_set(S, seg[2], tri[0] << 2 | 0, wkey(pos, 3));
  P2 v0 = S->pts[p[0]], v1 = S->pts[p[1]], v2 = S->pts[p[2]], v3 = S->pts[newp];
  if (encroached(v0, v3, v2, S->gc2, S->mode)) S->enc.a[sindex] = 0;
  if (encroached(v3, v1, v2, S->gc2, S->mode)) S->enc.a[nsub + tindex] = 0;
  neighbor[0] = S->nbr[tri[0] * 3 + triOri[0]];
  neighbor[1] = S->nbr[tri[0] * 3 + (triOri[0] + 1) % 3];
  neighbor[2] = S->nbr[tri[0] * 3 + (triOri[0] + 2) % 3];
  if (tri[2] == -1) {
    insert_tri(S, newp, p[2], p[0], tri[0], neighbor[2], -1, tri[1] << 2 | 1);
    insert_tri(S, newp, p[1], p[2], tri[1], neighbor[1], tri[0] << 2 | 2, -1);
  } else {
    insert_tri(S, newp, p[2], p[0], tri[0], neighbor[2], tri[2] << 2 | 2, tri[1] << 2 | 1);
    insert_tri(S, newp, p[1], p[2], tri[1], neighbor[1], tri[0] << 2 | 2, tri[3] << 2 | 1);
  }
  if (tri[2] != -1) {
    ts_set(&S->ts[tri[2]], TS_CHECK, 1);
    ts_set(&S->ts[tri[2]], TS_FLIP, 1);
    ts_setflipori(&S->ts[tri[2]], 0);
    ts_set(&S->ts[tri[3]], TS_NOTNULL, 1);
    ts_set(&S->ts[tri[3]], TS_CHECK, 1);
    ts_set(&S->ts[tri[3]], TS_FLIP, 1);
    ts_setflipori(&S->ts[tri[3]], 0);
    for (int i = 0; i < 3; i++) seg[i] = S->t2s[3 * tri[2] + (triOri[1] + i) % 3];
    S->t2s[3 * tri[2]] = seg[1];
    S->t2s[3 * tri[2] + 1] = -1;
    S->t2s[3 * tri[2] + 2] = seg[0];
    S->t2s[3 * tri[3]] = seg[2];
    S->t2s[3 * tri[3] + 1] = nsub + tindex;
    S->t2s[3 * tri[3] + 2] = -1;
    if (seg[1] != -1) s2t_set(S, seg[1], tri[2] << 2 | 0, wkey(pos, 4));
    if (seg[2] != -1) s2t_set(S, seg[2], tri[3] << 2 | 0, wkey(pos, 5));
    for (int i = 0; i < 3; i++) p[i] = S->tri[tri[2] * 3 + (triOri[1] + i + 1) % 3];
    v0 = S->pts[p[0]];
    v1 = S->pts[p[1]];
    v2 = S->pts[p[2]];
    v3 = S->pts[newp];
    if (encroached(v0, v3, v2, S->gc2, S->mode)) S->enc.a[nsub + tindex] = 0;
    if (encroached(v3, v1, v2, S->gc2, S->mode)) S->enc.a[sindex] = 0;
    neighbor[0] = S->nbr[tri[2] * 3 + triOri[1]];
    neighbor[1] = S->nbr[tri[2] * 3 + (triOri[1] + 1) % 3];
    neighbor[2] = S->nbr[tri[2] * 3 + (triOri[1] + 2) % 3];
    insert_tri(S, newp, p[1], p[2], tri[2], neighbor[1], tri[3] << 2 | 2, tri[0] << 2 | 1);
    insert_tri(S, newp, p[2], p[0], tri[3], neighbor[2], tri[1] << 2 | 2, tri[2] << 2 | 1);
  }
  imarker[tindex] = -1;
  S->midpoints_inserted++;
}

/* The outer-edge relinking shared by kernelUpdateMidNeighbors (2929-3070)
 * and kernelUpdateSteinerNeighbors (4902-5059): edge 0 of each new triangle
 * faces outward. */
static void relink_outer(St *S, const int *tri, int iteration) {
  for (int i = 0; i < iteration; i++) {
    int curTri = tri[i];
    int seg = S->t2s[3 * curTri + 0];
    int pOppTri = S->nbr[curTri * 3 + 0];
    int pOpp = dtri(pOppTri), pOri = dori(pOppTri);
    if (pOppTri < 0) {
      if (seg != -1) {
        S->enc.a[seg] = -1;
        P2 v0 = S->pts[S->tri[3 * curTri + 1]], v1 = S->pts[S->tri[3 * curTri + 2]];
        P2 v2 = S->pts[S->tri[3 * curTri]];
        if (encroached(v0, v1, v2, S->gc2, S->mode)) S->enc.a[seg] = 0;
      }
      continue;
    }
    if (ts_flipori(S->ts[pOpp]) == 15) {
      S->nbr[pOpp * 3 + pOri] = etri(curTri, 0);
      if (seg != -1) {
        S->enc.a[seg] = -1;
        P2 v0 = S->pts[S->tri[3 * curTri + 1]], v1 = S->pts[S->tri[3 * curTri + 2]];
        P2 v2 = S->pts[S->tri[3 * curTri]], v3 = S->pts[S->tri[3 * pOpp + pOri]];
        if (encroached(v0, v1, v2, S->gc2, S->mode))
          S->enc.a[seg] = 0;
        else if (encroached(v1, v0, v3, S->gc2, S->mode))
          S->enc.a[seg] = 0;
      }
    } else {
      int p0 = S->tri[curTri * 3 + 1], p1 = S->tri[curTri * 3 + 2];
      for (int j = 0; j < 3; j++) {
        int neighbor = (j == 0) ? pOpp : dtri(S->nbr[pOpp * 3 + j]);
        if (neighbor > -1) {
          int p2 = S->tri[neighbor * 3 + 1], p3 = S->tri[neighbor * 3 + 2];
          if (p0 == p3 && p1 == p2) {
            S->nbr[neighbor * 3 + 0] = etri(curTri, 0);
            if (seg != -1) {
              S->enc.a[seg] = -1;
              P2 v0 = S->pts[S->tri[3 * curTri + 1]], v1 = S->pts[S->tri[3 * curTri + 2]];
              P2 v2 = S->pts[S->tri[3 * curTri]], v3 = S->pts[S->tri[3 * neighbor + 0]];
              if (encroached(v0, v1, v2, S->gc2, S->mode))
                S->enc.a[seg] = 0;
              else if (encroached(v1, v0, v3, S->gc2, S->mode))
                S->enc.a[seg] = 0;
            }
            break;
          }
        }
      }
    }
  }
}

/* kernelUpdateMidNeighbors, refine.cu:2929-3070 */
static void update_mid_neighbors(St *S, int tindex, const int *imarker, const int *enclist) {
  if (imarker[tindex] != -1) return;
  int sindex = enclist[tindex];
  int tri[4], iteration;
  int otri = S->s2t.a[sindex];
  tri[0] = dtri(otri);
  tri[1] = dtri(S->nbr[3 * tri[0] + 2]);
  otri = S->nbr[3 * tri[0] + 1];
  iteration = (otri == -1) ? 2 : 4;
  tri[2] = dtri(otri);
  tri[3] = dtri(S->nbr[3 * tri[1] + 2]);
  relink_outer(S, tri, iteration);
}

/* splitEncsegs, refine.cu:3180-3778 */
static void split_encsegs(St *S) {
  IV *enclist = &S->l0, *imark = &S->l1, *ilist = &S->l2;
  long long outer = 0;
  for (;;) {
    enclist->n = 0;
    for (int s = 0; s < S->last_subseg; ++s)
      if (S->enc.a[s] >= 0) iv_push(enclist, s);
    int nenc = (int)enclist->n;
    if (nenc == 0) break;
    if (S->max_rounds && ++outer > S->max_rounds) {
      S->err = -2;
      return;
    }
    /* delete free Steiner points inside diametral circles */
    iv_resize(imark, 0, 0);
    for (int k = 0; k < nenc; ++k) iv_push(imark, enclist->a[k]);
    long long inner = 0;
    for (;;) {
      ilist->n = 0;
      for (long k = 0; k < imark->n; ++k)
        if (imark->a[k] >= 0) iv_push(ilist, imark->a[k]);
      int ndel = (int)ilist->n;
      if (ndel == 0) break;
      if (S->max_rounds && ++inner > S->max_rounds) {
        S->err = -2;
        return;
      }
      imark->n = ndel;
      for (int k = 0; k < ndel; ++k) mark_redundant_points(S, k, imark->a, ilist->a);
      flip_flop(S, S->last_triangle);
      if (S->err) return;
    }
    ensure_slots(S, nenc, 2 * nenc);
    iv_resize(&S->s2t, S->last_subseg + nenc, 0);
    iv_resize(&S->s2seg, S->last_subseg + nenc, 0);
    iv_resize(&S->enc, S->last_subseg + nenc, -1);
    iv_resize(imark, 0, 0);
    for (int k = 0; k < nenc; ++k) iv_push(imark, enclist->a[k]);
    long long mids_iter = 0;
    for (;;) {
      ilist->n = 0;
      for (int k = 0; k < nenc; ++k)
        if (imark->a[k] >= 0) iv_push(ilist, k);
      int nmid = (int)ilist->n;
      if (nmid == 0) break;
      if (S->max_rounds && ++mids_iter > 64 * S->max_rounds) {
        S->err = -2;
        return;
      }
      /* kernelResetMidInsertionMarker, refine.cu:2492-2542 */
      for (int k = 0; k < nmid; ++k) {
        int sindex = imark->a[ilist->a[k]];
        int otri = S->s2t.a[sindex];
        int t = dtri(otri), o = dori(otri);
        S->tmark[t] = MAXINT_REF;
        ts_setflipori(&S->ts[t], 15);
        for (int i = 0; i < 3; i++) {
          int n = dtri(S->nbr[3 * t + i]);
          if (n != -1) ts_setflipori(&S->ts[n], 15);
        }
        otri = S->nbr[3 * t + o];
        if (otri != -1) {
          t = dtri(otri);
          S->tmark[t] = MAXINT_REF;
          ts_setflipori(&S->ts[t], 15);
          for (int i = 0; i < 3; i++) {
            int n = dtri(S->nbr[3 * t + i]);
            if (n != -1) ts_setflipori(&S->ts[n], 15);
          }
        }
      }
      /* kernelMarkMidInsertion, refine.cu:2544-2579 */
      for (int k = 0; k < nmid; ++k) {
        int sindex = imark->a[ilist->a[k]];
        int otri = S->s2t.a[sindex];
        int t = dtri(otri), o = dori(otri);
        amin(&S->tmark[t], sindex);
        otri = S->nbr[3 * t + o];
        if (otri != -1) amin(&S->tmark[dtri(otri)], sindex);
      }
      /* every thread of kernelInsertMidPoints reads subseg2tri[sindex] before
       * any winner rewrites it (a losing thread may otherwise read a winner's
       * fresh triangle) */
      int *snap = (int *)malloc(sizeof(int) * (nmid + 1));
      for (int k = 0; k < nmid; ++k) snap[k] = S->s2t.a[imark->a[ilist->a[k]]];
      s2t_begin(S);
      for (int k = 0; k < nmid; ++k) insert_midpoint(S, k, ilist->a[k], imark->a, S->last_subseg, snap[k]);
      free(snap);
      for (int k = 0; k < nmid; ++k) update_mid_neighbors(S, ilist->a[k], imark->a, enclist->a);
    }
    consume_slots(S, nenc, 2 * nenc);
    S->last_subseg += nenc;
    flip_flop(S, S->last_triangle);
    if (S->err) return;
  }
}

/* ---------------- bad triangles (refine.cu:376-570) ---------------- */
/* twice the area of triangle (a, b, c), as the CUDA kernels compute it */
static double area2(P2 a, P2 b, P2 c) { return fabs((b.x - a.x) * (c.y - a.y) - (b.y - a.y) * (c.x - a.x)); }

/* kernelMarkBadTriangles with an optional area bound (no counterpart in the
 * reference): a triangle larger than max_area is bad whatever its angles. */
static void mark_bad_angle(St *S, int index);
static void mark_bad(St *S, int index) {
  unsigned char *ts = &S->ts[index];
  if (!(*ts & TS_CHECK)) return;
  mark_bad_angle(S, index);
  if (S->max_area > 0.0 && !(*ts & TS_BAD)) {
    const int *p = &S->tri[3 * index];
    if (0.5 * area2(S->pts[p[0]], S->pts[p[1]], S->pts[p[2]]) > S->max_area) ts_set(ts, TS_BAD, 1);
  }
}
static void mark_bad_angle(St *S, int index) {
  unsigned char *ts = &S->ts[index];
  ts_set(ts, TS_CHECK, 0);
  ts_set(ts, TS_NOTNULL, 1);
  int p[3] = {S->tri[3 * index], S->tri[3 * index + 1], S->tri[3 * index + 2]};
  P2 v[3] = {S->pts[p[0]], S->pts[p[1]], S->pts[p[2]]};
  int shortest;
  double c2 = smallest_angle(v[0], v[1], v[2], &shortest);
  if (c2 <= S->gc2) {
    ts_set(ts, TS_BAD, 0);
    return;
  }
  if (S->t2s[3 * index + shortest] == -1) {
    int eOrg = p[(shortest + 1) % 3], eDest = p[(shortest + 2) % 3];
    if ((S->ps[eOrg] & PS_SEGSPLIT) && (S->ps[eDest] & PS_SEGSPLIT)) {
      int s1 = -1, s2 = -1, curTri, curOri;
      long guard = 0;
      curTri = index;
      curOri = shortest;
      do {
        int otri = S->nbr[3 * curTri + curOri];
        curTri = dtri(otri);
        curOri = (dori(otri) + 1) % 3;
        if (curTri < 0 || ++guard > 1000000) {
          S->err = -5;
          return;
        }
        s1 = S->t2s[3 * curTri + curOri];
      } while (s1 == -1);
      curTri = index;
      curOri = shortest;
      do {
        int otri = S->nbr[3 * curTri + curOri];
        curTri = dtri(otri);
        curOri = (dori(otri) + 2) % 3;
        if (curTri < 0 || ++guard > 2000000) {
          S->err = -5;
          return;
        }
        s2 = S->t2s[3 * curTri + curOri];
      } while (s2 == -1);
      s1 = S->s2seg.a[s1];
      s2 = S->s2seg.a[s2];
      int pOrg1 = S->segs[2 * s1], pDest1 = S->segs[2 * s1 + 1];
      int pOrg2 = S->segs[2 * s2], pDest2 = S->segs[2 * s2 + 1];
      int common = -1;
      if (pOrg1 == pOrg2 || pOrg1 == pDest2)
        common = pOrg1;
      else if (pDest1 == pOrg2 || pDest1 == pDest2)
        common = pDest1;
      if (common != -1) {
        P2 vOrg = v[(shortest + 1) % 3], vDest = v[(shortest + 2) % 3], vCom = S->pts[common];
        double d1 = madd(vCom.x - vOrg.x, vCom.x - vOrg.x, (vCom.y - vOrg.y) * (vCom.y - vOrg.y));
        double d2 = madd(vCom.x - vDest.x, vCom.x - vDest.x, (vCom.y - vDest.y) * (vCom.y - vDest.y));
        if ((d1 < 1.001 * d2) && (d1 > 0.999 * d2)) {
          ts_set(ts, TS_BAD, 0);
          return;
        }
      }
    }
  }
  ts_set(ts, TS_BAD, 1);
}

/* ---------------- Steiner insertion (refine.cu:3870-5547) ---------------- */
typedef struct {
  int a[LS_REF];
  int size;
} MyList;
static int ml_find(const MyList *l, int v) {
  for (int i = 0; i < l->size; i++)
    if (l->a[i] == v) return 1;
  return 0;
}
static int ml_push(MyList *l, int v) {
  if (l->size == LS_REF) return 0;
  l->a[l->size++] = v;
  return 1;
}

/* the cavity walk shared by kernelMarkCavities (4237-4368) and
 * kernelCheckCavities (4422-4547).  check == 0: claim with atomicMin;
 * check == 1: verify ownership.  Returns -1 on overflow (mark) or on a lost
 * triangle (check), else 0. */
static int cavity(St *S, int sink, int direction, P2 cc, int badIndex, int check) {
  MyList region, loop;
  region.size = loop.size = 0;
  int cur = sink;
  for (;;) {
    if (!ml_find(&region, cur)) {
      if (!ml_push(&region, cur)) return check ? 0 : -1;
      if (!ml_push(&loop, cur)) return check ? 0 : -1;
      if (check) {
        if (S->tmark[cur] != badIndex) return -1;
      } else {
        amin(&S->tmark[cur], badIndex);
      }
    }
    int recursive = 0, nIdx = -1;
    for (int i = 0; i < 3; i++) {
      if (cur == sink) {
        if (direction == 3 && S->t2s[3 * cur + i] != -1) continue;
        if (direction < 3 && S->t2s[3 * cur + i] != -1 && i != direction) continue;
      } else if (S->t2s[3 * cur + i] != -1)
        continue;
      int neighbor = S->nbr[3 * cur + i];
      if (neighbor == -1) continue;
      nIdx = dtri(neighbor);
      if (ml_find(&region, nIdx)) continue;
      P2 v0 = S->pts[S->tri[3 * nIdx]], v1 = S->pts[S->tri[3 * nIdx + 1]], v2 = S->pts[S->tri[3 * nIdx + 2]];
      double r = incircle_pair(v0, v1, v2, cc);
      if (r > 0) {
        recursive = 1;
        break;
      }
    }
    if (recursive)
      cur = nIdx;
    else {
      if (loop.size > 0) loop.size--;
      if (loop.size == 0) break;
      cur = loop.a[loop.size - 1];
    }
  }
  return 0;
}

/* kernelLocateSinkPoints, refine.cu:3908-4184 */
static int locate_sink(St *S, int index, P2 cc) {
  int curTri = index, curOri = 0;
  int checkNeighbor = 0, split = 0, direction_dart = 3;
  P2 v[3] = {S->pts[S->tri[3 * curTri]], S->pts[S->tri[3 * curTri + 1]], S->pts[S->tri[3 * curTri + 2]]};
  double det0 = orient_ref(v[0], v[1], cc), det1 = orient_ref(v[1], v[2], cc), det2 = orient_ref(v[2], v[0], cc);
  if (det0 <= 0) {
    if (det0 == 0 || S->t2s[3 * index + 2] != -1) split = 1;
    direction_dart = 2;
  } else if (det1 <= 0) {
    if (det1 == 0 || S->t2s[3 * index + 0] != -1) split = 1;
    direction_dart = 0;
  } else if (det2 <= 0) {
    if (det2 == 0 || S->t2s[3 * index + 1] != -1) split = 1;
    direction_dart = 1;
  }
  if (!split && direction_dart != 3) {
    int neighbor = S->nbr[3 * curTri + direction_dart];
    if (neighbor < 0) {
      checkNeighbor = 0;
      split = 1;
    } else {
      curTri = dtri(neighbor);
      curOri = dori(neighbor);
      checkNeighbor = 1;
    }
  }
  long guard = 0;
  while (checkNeighbor) {
    if (++guard > 4 * S->tcap + 16) {
      S->err = -3;
      break;
    }
    v[0] = S->pts[S->tri[3 * curTri]];
    v[1] = S->pts[S->tri[3 * curTri + 1]];
    v[2] = S->pts[S->tri[3 * curTri + 2]];
    direction_dart = 3;
    int pOrg = (curOri + 1) % 3, pDest = (curOri + 2) % 3, pApex = curOri;
    double detLeft = orient_ref(v[pDest], v[pApex], cc);
    double detRight = orient_ref(v[pApex], v[pOrg], cc);
    int moveleft;
    if (detLeft < 0.0) {
      if (detRight < 0.0)
        moveleft = madd(v[(curOri + 2) % 3].x - v[(curOri + 1) % 3].x, cc.x - v[curOri].x,
                        (v[(curOri + 2) % 3].y - v[(curOri + 1) % 3].y) * (cc.y - v[curOri].y)) > 0.0;
      else
        moveleft = 1;
    } else {
      if (detRight < 0.0)
        moveleft = 0;
      else {
        if (detLeft == 0.0) {
          split = 1;
          direction_dart = (curOri + 1) % 3;
          break;
        }
        if (detRight == 0.0) {
          split = 1;
          direction_dart = (curOri + 2) % 3;
          break;
        }
        break;
      }
    }
    direction_dart = moveleft ? (curOri + 1) % 3 : (curOri + 2) % 3;
    int neighbor = S->nbr[3 * curTri + direction_dart];
    if (neighbor < 0 || S->t2s[3 * curTri + direction_dart] != -1) {
      split = 1;
      break;
    }
    curTri = dtri(neighbor);
    curOri = dori(neighbor);
  }
  amin(&S->tmark[curTri], index);
  if (split) {
    int neighbor = S->nbr[3 * curTri + direction_dart];
    if (neighbor != -1) amin(&S->tmark[dtri(neighbor)], index);
  }
  return (curTri << 2) | direction_dart;
}

/* kernelInsertSteinerPoints, refine.cu:4651-4900 */
static void insert_steiner(St *S, int pos, int tindex, const int *sinks, const P2 *center) {
  int index = sinks[tindex] >> 2, direction = sinks[tindex] & 3;
  if (direction != 3 && S->t2s[3 * index + direction] != -1) return;
  int tri[4], p[3], neighbor[3], seg[3];
  int newp = new_point_slot(S, pos);
  S->ps[newp] = PS_STEINER | PS_NEW;
  int nt1 = new_tri_slot(S, 2 * pos), nt2 = new_tri_slot(S, 2 * pos + 1);
  tri[0] = index;
  S->steiner_inserted++;
  if (direction == 3) {
    tri[1] = nt1;
    tri[2] = nt2;
    S->ts[tri[1]] = 0;
    S->ts[tri[2]] = 0;
    ts_set(&S->ts[tri[0]], TS_CHECK, 1);
    ts_set(&S->ts[tri[0]], TS_FLIP, 1);
    ts_setflipori(&S->ts[tri[0]], 0);
    for (int k = 1; k <= 2; ++k) {
      ts_set(&S->ts[tri[k]], TS_NOTNULL, 1);
      ts_set(&S->ts[tri[k]], TS_CHECK, 1);
      ts_set(&S->ts[tri[k]], TS_FLIP, 1);
      ts_setflipori(&S->ts[tri[k]], 0);
    }
    S->pts[newp] = center[tindex];
    for (int i = 0; i < 3; i++) p[i] = S->tri[tri[0] * 3 + (i + 1) % 3];
    for (int i = 0; i < 3; i++) seg[i] = S->t2s[3 * tri[0] + i];
    S->t2s[3 * tri[0]] = seg[0];
    S->t2s[3 * tri[0] + 1] = -1;
    S->t2s[3 * tri[0] + 2] = -1;
    S->t2s[3 * tri[1]] = seg[1];
    S->t2s[3 * tri[1] + 1] = -1;
    S->t2s[3 * tri[1] + 2] = -1;
    S->t2s[3 * tri[2]] = seg[2];
    S->t2s[3 * tri[2] + 1] = -1;
    S->t2s[3 * tri[2] + 2] = -1;
    if (seg[0] != -1) s2t_set(S, seg[0], tri[0] << 2 | 0, wkey(pos, 0));
    if (seg[1] != -1) s2t_set(S, seg[1], tri[1] << 2 | 0, wkey(pos, 1));
    if (seg[2] != -1) s2t_set(S, seg[2], tri[2] << 2 | 0, wkey(pos, 2));
    for (int i = 0; i < 3; i++) neighbor[i] = S->nbr[tri[0] * 3 + i];
    insert_tri(S, newp, p[0], p[1], tri[0], neighbor[0], tri[1] << 2 | 2, tri[2] << 2 | 1);
    insert_tri(S, newp, p[1], p[2], tri[1], neighbor[1], tri[2] << 2 | 2, tri[0] << 2 | 1);
    insert_tri(S, newp, p[2], p[0], tri[2], neighbor[2], tri[0] << 2 | 2, tri[1] << 2 | 1);
  } else {
    int triOri[2];
    triOri[0] = direction;
    int otri = S->nbr[3 * tri[0] + triOri[0]];
    triOri[1] = dori(otri);
    tri[1] = nt1;
    tri[2] = dtri(otri);
    tri[3] = nt2;
    S->ts[tri[1]] = 0;
    S->ts[tri[3]] = 0;
    ts_set(&S->ts[tri[0]], TS_CHECK, 1);
    ts_set(&S->ts[tri[0]], TS_FLIP, 1);
    ts_setflipori(&S->ts[tri[0]], 0);
    ts_set(&S->ts[tri[1]], TS_NOTNULL, 1);
    ts_set(&S->ts[tri[1]], TS_CHECK, 1);
    ts_set(&S->ts[tri[1]], TS_FLIP, 1);
    ts_setflipori(&S->ts[tri[1]], 0);
    S->pts[newp] = center[tindex];
    for (int i = 0; i < 3; i++) p[i] = S->tri[tri[0] * 3 + (triOri[0] + i + 1) % 3];
    for (int i = 0; i < 3; i++) seg[i] = S->t2s[3 * tri[0] + (triOri[0] + i) % 3];
    S->t2s[3 * tri[0]] = seg[2];
    S->t2s[3 * tri[0] + 1] = seg[0];
    S->t2s[3 * tri[0] + 2] = -1;
    S->t2s[3 * tri[1]] = seg[1];
    S->t2s[3 * tri[1] + 1] = -1;
    S->t2s[3 * tri[1] + 2] = seg[0];
    if (seg[1] != -1) s2t_set(S, seg[1], tri[1] << 2 | 0, wkey(pos, 3));
    if (seg[2] != -1) s2t_set(S, seg[2], tri[0] << 2 | 0, wkey(pos, 4));
    neighbor[0] = S->nbr[tri[0] * 3 + triOri[0]];
    neighbor[1] = S->nbr[tri[0] * 3 + (triOri[0] + 1) % 3];
    neighbor[2] = S->nbr[tri[0] * 3 + (triOri[0] + 2) % 3];
    if (tri[2] == -1) {
      insert_tri(S, newp, p[2], p[0], tri[0], neighbor[2], -1, tri[1] << 2 | 1);
      insert_tri(S, newp, p[1], p[2], tri[1], neighbor[1], tri[0] << 2 | 2, -1);
    } else {
      insert_tri(S, newp, p[2], p[0], tri[0], neighbor[2], tri[2] << 2 | 2, tri[1] << 2 | 1);
      insert_tri(S, newp, p[1], p[2], tri[1], neighbor[1], tri[0] << 2 | 2, tri[3] << 2 | 1);
    }
    if (tri[2] != -1) {
      ts_set(&S->ts[tri[2]], TS_CHECK, 1);
      ts_set(&S->ts[tri[2]], TS_FLIP, 1);
      ts_setflipori(&S->ts[tri[2]], 0);
      ts_set(&S->ts[tri[3]], TS_NOTNULL, 1);
      ts_set(&S->ts[tri[3]], TS_CHECK, 1);
      ts_set(&S->ts[tri[3]], TS_FLIP, 1);
      ts_setflipori(&S->ts[tri[3]], 0);
      for (int i = 0; i < 3; i++) p[i] = S->tri[tri[2] * 3 + (triOri[1] + i + 1) % 3];
      for (int i = 0; i < 3; i++) seg[i] = S->t2s[3 * tri[2] + (triOri[1] + i) % 3];
      S->t2s[3 * tri[2]] = seg[1];
      S->t2s[3 * tri[2] + 1] = -1;
      S->t2s[3 * tri[2] + 2] = seg[0];
      S->t2s[3 * tri[3]] = seg[2];
      S->t2s[3 * tri[3] + 1] = seg[0];
      S->t2s[3 * tri[3] + 2] = -1;
      if (seg[1] != -1) s2t_set(S, seg[1], tri[2] << 2 | 0, wkey(pos, 5));
      if (seg[2] != -1) s2t_set(S, seg[2], tri[3] << 2 | 0, wkey(pos, 6));
      neighbor[0] = S->nbr[tri[2] * 3 + triOri[1]];
      neighbor[1] = S->nbr[tri[2] * 3 + (triOri[1] + 1) % 3];
      neighbor[2] = S->nbr[tri[2] * 3 + (triOri[1] + 2) % 3];
      insert_tri(S, newp, p[1], p[2], tri[2], neighbor[1], tri[3] << 2 | 2, tri[0] << 2 | 1);
      insert_tri(S, newp, p[2], p[0], tri[3], neighbor[2], tri[1] << 2 | 2, tri[2] << 2 | 1);
    }
  }
}

/* kernelUpdateSteinerNeighbors, refine.cu:4902-5059 */
static void update_steiner_neighbors(St *S, int tindex, const int *sinks) {
  int index = sinks[tindex] >> 2, direction = sinks[tindex] & 3;
  if (direction != 3 && ts_flipori(S->ts[index]) == 15) return;
  int tri[4], iteration;
  if (direction == 3) {
    iteration = 3;
    tri[0] = index;
    tri[1] = dtri(S->nbr[3 * tri[0] + 1]);
    tri[2] = dtri(S->nbr[3 * tri[0] + 2]);
  } else {
    tri[0] = index;
    tri[1] = dtri(S->nbr[3 * tri[0] + 2]);
    int otri = S->nbr[3 * tri[0] + 1];
    if (otri == -1)
      iteration = 2;
    else {
      iteration = 4;
      tri[2] = dtri(otri);
      tri[3] = dtri(S->nbr[3 * tri[1] + 2]);
    }
  }
  relink_outer(S, tri, iteration);
}

/* splitTriangles, refine.cu:5107-5547 */
static void split_triangles(St *S, const IV *bad, int offconstant, int offcenter) {
  int nbad = (int)bad->n;
  int *imark = (int *)malloc(sizeof(int) * (nbad + 1));
  int *ilist = (int *)malloc(sizeof(int) * (nbad + 1));
  int *sinks = (int *)malloc(sizeof(int) * (nbad + 1));
  P2 *center = (P2 *)malloc(sizeof(P2) * (nbad + 1));
  memcpy(imark, bad->a, sizeof(int) * nbad);
  memcpy(ilist, bad->a, sizeof(int) * nbad);
  for (int k = 0; k < nbad; ++k) {
    int t = ilist[k];
    P2 v0 = S->pts[S->tri[3 * t]], v1 = S->pts[S->tri[3 * t + 1]], v2 = S->pts[S->tri[3 * t + 2]];
    center[k] = circumcenter(v0, v1, v2, (double)offconstant, offcenter);
  }
  for (int t = 0; t < S->last_triangle; ++t) S->tmark[t] = MAXINT_REF;
  for (int k = 0; k < nbad; ++k) {
    sinks[k] = -1;
    if (!(S->ts[ilist[k]] & TS_BAD)) continue;
    sinks[k] = locate_sink(S, ilist[k], center[k]);
  }
  /* kernelRemoveLosers, refine.cu:4186-4235 */
  for (int k = 0; k < nbad; ++k) {
    if (imark[k] < 0) continue;
    int sink = sinks[k] >> 2, index = ilist[k], dir = sinks[k] & 3;
    if (S->tmark[sink] != index) {
      imark[k] = -1;
      continue;
    }
    if (dir != 3) {
      int nb = S->nbr[3 * sink + dir];
      if (nb != -1 && S->tmark[dtri(nb)] != index) imark[k] = -1;
    }
  }
  for (int t = 0; t < S->last_triangle; ++t) S->tmark[t] = MAXINT_REF;
  for (int k = 0; k < nbad; ++k) {
    if (imark[k] < 0) continue;
    int badIndex = ilist[k];
    if (cavity(S, sinks[k] >> 2, sinks[k] & 3, center[k], badIndex, 0) < 0) ilist[k] = negate_ref(badIndex);
  }
  for (int k = 0; k < nbad; ++k) {
    if (imark[k] < 0) continue;
    int badIndex = ilist[k];
    if (badIndex < 0) continue;
    if (cavity(S, sinks[k] >> 2, sinks[k] & 3, center[k], badIndex, 1) < 0) imark[k] = -1;
  }
  int nst = 0;
  for (int k = 0; k < nbad; ++k)
    if (imark[k] >= 0) ilist[nst++] = k;
  /* on-segment centres, refine.cu:5249-5257 */
  IV *enclist = &S->l0;
  iv_resize(enclist, 0, 0);
  iv_resize(enclist, S->last_subseg, -1);
  for (int w = 0; w < nst; ++w) {
    int tindex = ilist[w];
    int index = sinks[tindex] >> 2, dir = sinks[tindex] & 3;
    if (dir != 3) {
      int sg = S->t2s[3 * index + dir];
      if (sg != -1) enclist->a[sg] = 0;
    }
  }
  ensure_slots(S, nst, 2 * nst);
  /* kernelResetSteinerInsertionMarker, refine.cu:4601-4649 */
  for (int w = 0; w < nst; ++w) {
    int tindex = ilist[w];
    int index = sinks[tindex] >> 2, dir = sinks[tindex] & 3;
    ts_setflipori(&S->ts[index], 15);
    for (int i = 0; i < 3; i++) {
      int n = dtri(S->nbr[3 * index + i]);
      if (n != -1) ts_setflipori(&S->ts[n], 15);
    }
    if (dir != 3) {
      int otri = S->nbr[3 * index + dir];
      if (otri != -1) {
        int t = dtri(otri);
        ts_setflipori(&S->ts[t], 15);
        for (int i = 0; i < 3; i++) {
          int n = dtri(S->nbr[3 * t + i]);
          if (n != -1) ts_setflipori(&S->ts[n], 15);
        }
      }
    }
  }
  s2t_begin(S);
  for (int w = 0; w < nst; ++w) insert_steiner(S, w, ilist[w], sinks, center);
  for (int w = 0; w < nst; ++w) update_steiner_neighbors(S, ilist[w], sinks);
  consume_slots(S, nst, 2 * nst);
  flip_flop(S, S->last_triangle);
  /* kernelUpdateSteinerOnsegs, refine.cu:5091-5105 */
  for (int s = 0; s < S->last_subseg; ++s)
    if (enclist->a[s] >= 0) S->enc.a[s] = 1;
  free(imark);
  free(ilist);
  free(sinks);
  free(center);
}

/* ---------------- compaction (refine.cu:5758-6484) ---------------- */
static int compact_tris(St *S, int ntri, int nsub) {
  int *valid = (int *)malloc(sizeof(int) * (ntri + 1)), *prefix = (int *)malloc(sizeof(int) * (ntri + 1));
  int run = 0;
  for (int t = 0; t < ntri; ++t) {
    valid[t] = ts_null(S->ts[t]) ? 0 : 1;
    prefix[t] = run;
    run += valid[t];
  }
  int newn = run;
  if (newn == ntri) {
    free(valid);
    free(prefix);
    return newn;
  }
  int offset = prefix[newn];
  int *empty = valid; /* the reference reuses the valid array */
  for (int t = 0; t < ntri; ++t)
    if (ts_null(S->ts[t])) empty[t - prefix[t]] = t;
  for (int t = 0; t < ntri; ++t) {
    if (ts_null(S->ts[t])) {
      prefix[t] = -1;
      continue;
    }
    int value;
    if (t < newn)
      value = t;
    else {
      value = empty[prefix[t] - offset];
      for (int i = 0; i < 3; i++) {
        S->tri[value * 3 + i] = S->tri[t * 3 + i];
        S->nbr[value * 3 + i] = S->nbr[t * 3 + i];
      }
    }
    prefix[t] = value;
  }
  for (int t = 0; t < newn; ++t)
    for (int i = 0; i < 3; ++i)
      if (S->nbr[3 * t + i] >= 0) S->nbr[3 * t + i] = etri(prefix[dtri(S->nbr[3 * t + i])], dori(S->nbr[3 * t + i]));
  for (int t = 0; t < ntri; ++t)
    if (prefix[t] != -1) S->ts[prefix[t]] = S->ts[t];
  for (int s = 0; s < nsub; ++s) {
    int o = S->s2t.a[s];
    S->s2t.a[s] = etri(prefix[dtri(o)], dori(o));
  }
  free(valid);
  free(prefix);
  return newn;
}
static int compact_points(St *S, int ntri, int npts) {
  int *valid = (int *)malloc(sizeof(int) * (npts + 1)), *prefix = (int *)malloc(sizeof(int) * (npts + 1));
  int run = 0;
  for (int i = 0; i < npts; ++i) {
    valid[i] = (S->ps[i] & PS_DELETED) ? 0 : 1;
    prefix[i] = run;
    run += valid[i];
  }
  int newn = run;
  if (newn == npts) {
    free(valid);
    free(prefix);
    return newn;
  }
  int offset = prefix[newn];
  int *empty = valid;
  for (int i = 0; i < npts; ++i)
    if (S->ps[i] & PS_DELETED) empty[i - prefix[i]] = i;
  for (int i = 0; i < npts; ++i) {
    if (S->ps[i] & PS_DELETED) {
      prefix[i] = -1;
      continue;
    }
    int value;
    if (i < newn)
      value = i;
    else {
      value = empty[prefix[i] - offset];
      S->pts[value] = S->pts[i];
    }
    prefix[i] = value;
  }
  for (int t = 0; t < ntri; ++t)
    for (int k = 0; k < 3; ++k) S->tri[3 * t + k] = prefix[S->tri[3 * t + k]];
  for (int i = 0; i < npts; ++i)
    if (prefix[i] != -1) S->ps[prefix[i]] = S->ps[i];
  free(valid);
  free(prefix);
  return newn;
}

/* ---------------- driver (refine.cu:6500-7139) ---------------- */
static int find_incident_ori(const int *tri, int t1, int t2) { /* findIncidentOri, 35-93 */
  if (t1 < 0 || t2 < 0) return -1;
  int inc0 = -1, inc1 = -1, count = 0;
  const int *a = tri + 3 * t1, *b = tri + 3 * t2;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      if (a[i] == b[j]) {
        if (count == 0) {
          inc0 = j;
          count += 1;
          continue;
        } else {
          inc1 = j;
          break;
        }
      }
  if (inc0 == -1 || inc1 == -1) return -1;
  int differ = inc0 - inc1, index;
  if (differ == -1 || differ == 2)
    index = inc0;
  else
    index = inc1;
  if (index == 0) return 2;
  if (index == 1) return 0;
  if (index == 2) return 1;
  return -1;
}

int gqm_oracle_refine(int np, const double *pts, int nt, const int *tri, const int *nbr, int ns, const int *segs,
                      double theta, int policy, int mode, long long max_rounds, gqm_oracle_out *out) {
  return gqm_oracle_refine_gc(np, pts, nt, tri, nbr, ns, segs, theta, 0.0, policy, mode, max_rounds, out);
}

static double g_max_area = 0.0;
void gqm_oracle_set_max_area(double a) { g_max_area = a > 0.0 ? a : 0.0; }

int gqm_oracle_refine_gc(int np, const double *pts, int nt, const int *tri, const int *nbr, int ns,
                         const int *segs, double theta, double goodcos2, int policy, int mode, long long max_rounds,
                         gqm_oracle_out *out) {
  memset(out, 0, sizeof(*out));
  St Sv;
  St *S = &Sv;
  memset(S, 0, sizeof(*S));
  S->max_area = g_max_area;
  S->theta = theta;
  S->mode = mode;
  S->max_rounds = max_rounds;
  if (goodcos2 > 0.0) {
    S->gc2 = goodcos2;
  } else {  /* refine.cu:418-419 */
    double c = cos(theta * PI_REF / 180.0);
    S->gc2 = c * c;
  }
  S->pointblock = (int)(np * 0.5);
  S->triblock = 2 * S->pointblock;
  int offcenter = 0;
  double offc = 0.0;
  if (policy == 1) {
    offcenter = 1;
    double cg = cos(theta * PI_REF / 180);
    offc = 0.475 * sqrt((1.0 + cg) / (1.0 - cg));
  }
  int offconstant = (int)offc; /* splitTriangles takes an int (refine.cu:5132) */
  long presize = np + S->pointblock, tresize = nt + S->triblock;
  S->pcap = 0;
  S->tcap = 0;
  grow_points(S, presize);
  grow_tris(S, tresize);
  memcpy(S->pts, pts, sizeof(double) * 2 * np);
  for (int i = 0; i < np; ++i) S->ps[i] = 0;
  memcpy(S->tri, tri, sizeof(int) * 3 * nt);
  for (int t = 0; t < nt; ++t)
    for (int i = 0; i < 3; ++i) {
      int n = nbr[3 * t + i];
      S->nbr[3 * t + i] = etri(n, find_incident_ori(S->tri, t, n));
    }
  for (int t = 0; t < nt; ++t) S->ts[t] = TS_NOTNULL | TS_CHECK;
  S->segs = (int *)malloc(sizeof(int) * (2 * ns + 2));
  memcpy(S->segs, segs, sizeof(int) * 2 * ns);
  iv_resize(&S->s2t, ns, -1);
  iv_resize(&S->s2seg, ns, 0);
  for (int s = 0; s < ns; ++s) S->s2seg.a[s] = s;
  /* initSubsegs (refine.cu:5618-5747): triangle edge (p0,p1) is ori 2,
   * (p1,p2) ori 0, (p2,p0) ori 1; subseg2tri keeps the largest otri */
  {
    /* hash segments by unordered endpoint pair */
    long hsz = 1;
    while (hsz < 4L * ns + 8) hsz <<= 1;
    long long *hk = (long long *)malloc(sizeof(long long) * hsz);
    int *hv = (int *)malloc(sizeof(int) * hsz);
    for (long i = 0; i < hsz; ++i) hk[i] = -1;
    for (int s = 0; s < ns; ++s) {
      int a = segs[2 * s], b = segs[2 * s + 1];
      long long k = a < b ? ((long long)a << 32) | (unsigned)b : ((long long)b << 32) | (unsigned)a;
      unsigned long long h = (unsigned long long)k * 0x9E3779B97F4A7C15ull;
      long i = (long)(h >> 20) & (hsz - 1);
      while (hk[i] != -1) i = (i + 1) & (hsz - 1);
      hk[i] = k;
      hv[i] = s;
    }
    for (int t = 0; t < nt; ++t) {
      int p[3] = {tri[3 * t], tri[3 * t + 1], tri[3 * t + 2]};
      const int ed[3][3] = {{0, 1, 2}, {1, 2, 0}, {2, 0, 1}}; /* (u, w, ori) */
      for (int e = 0; e < 3; ++e) {
        int a = p[ed[e][0]], b = p[ed[e][1]], ori = ed[e][2];
        long long k = a < b ? ((long long)a << 32) | (unsigned)b : ((long long)b << 32) | (unsigned)a;
        unsigned long long h = (unsigned long long)k * 0x9E3779B97F4A7C15ull;
        long i = (long)(h >> 20) & (hsz - 1);
        while (hk[i] != -1) {
          if (hk[i] == k) {
            int s = hv[i];
            int ot = (t << 2) | ori;
            if (ot > S->s2t.a[s]) S->s2t.a[s] = ot;
            if (s > S->t2s[3 * t + ori]) S->t2s[3 * t + ori] = s;
          }
          i = (i + 1) & (hsz - 1);
        }
      }
    }
    free(hk);
    free(hv);
  }
  S->last_point = np;
  S->last_triangle = nt;
  S->last_subseg = ns;
  S->nempty_p = refresh_empty_points(S);
  S->nempty_t = refresh_empty_tris(S);
  /* markAllEncsegs, refine.cu:3105-3178 */
  iv_resize(&S->enc, ns, -1);
  for (int s = 0; s < ns; ++s) {
    S->enc.a[s] = -1;
    int otri = S->s2t.a[s];
    if (otri < 0) continue; /* a segment that is not an edge: the reference reads out of bounds */
    int t = dtri(otri), o = dori(otri);
    P2 vo = S->pts[S->tri[3 * t + (o + 1) % 3]], vd = S->pts[S->tri[3 * t + (o + 2) % 3]];
    P2 va = S->pts[S->tri[3 * t + o]];
    if (encroached(vo, vd, va, S->gc2, mode)) S->enc.a[s] = 0;
    otri = S->nbr[3 * t + o];
    if (otri != -1) {
      va = S->pts[S->tri[3 * dtri(otri) + dori(otri)]];
      if (encroached(vd, vo, va, S->gc2, mode)) S->enc.a[s] = 0;
    }
  }
  split_encsegs(S);
  int iteration = 0;
  IV bad = {0, 0, 0};
  while (!S->err) {
    /* updateActiveListToBadTriangles, refine.cu:499-570 */
    for (int t = 0; t < S->last_triangle; ++t) {
      unsigned char s = S->ts[t];
      if (!ts_null(s) && ((s & TS_CHECK) || (s & TS_BAD))) mark_bad(S, t);
    }
    if (S->err) break;
    bad.n = 0;
    for (int t = 0; t < S->last_triangle; ++t)
      if (!ts_null(S->ts[t]) && (S->ts[t] & TS_BAD)) iv_push(&bad, t);
    if (bad.n == 0) break;
    if (max_rounds && iteration >= max_rounds) {
      S->err = -2;
      break;
    }
    S->bad_total += bad.n;
    split_triangles(S, &bad, offconstant, offcenter);
    if (S->err) break;
    split_encsegs(S);
    /* updatePStatus2Old, refine.cu:3072-3095 */
    for (int i = 0; i < S->last_point; ++i)
      if (!(S->ps[i] & PS_DELETED)) S->ps[i] &= (unsigned char)~PS_NEW;
    iteration++;
  }
  free(bad.a);
  out->rounds = iteration;
  out->flip_steps = S->flip_steps;
  out->steiner_inserted = S->steiner_inserted;
  out->midpoints_inserted = S->midpoints_inserted;
  out->bad_total = S->bad_total;
  if (!S->err) {
    int ntri = compact_tris(S, S->last_triangle, S->last_subseg);
    int npts = compact_points(S, ntri, S->last_point);
    out->numberofpoints = npts;
    out->numberoftriangles = ntri;
    out->numberofsegments = S->last_subseg;
    out->pointlist = (double *)malloc(sizeof(double) * 2 * (npts + 1));
    memcpy(out->pointlist, S->pts, sizeof(double) * 2 * npts);
    out->trianglelist = (int *)malloc(sizeof(int) * 3 * (ntri + 1));
    memcpy(out->trianglelist, S->tri, sizeof(int) * 3 * ntri);
    out->neighborlist = (int *)malloc(sizeof(int) * 3 * (ntri + 1));
    for (long i = 0; i < 3L * ntri; ++i) out->neighborlist[i] = dtri(S->nbr[i]);
    out->segmentlist = (int *)malloc(sizeof(int) * 2 * (S->last_subseg + 1));
    for (int s = 0; s < S->last_subseg; ++s) { /* kernelCompactSegment, 6365-6388 */
      int o = S->s2t.a[s];
      int t = dtri(o), r = dori(o);
      out->segmentlist[2 * s] = S->tri[3 * t + (r + 1) % 3];
      out->segmentlist[2 * s + 1] = S->tri[3 * t + (r + 2) % 3];
    }
    out->pstatus = (unsigned char *)malloc((size_t)npts + 1);
    memcpy(out->pstatus, S->ps, (size_t)npts);
    out->tstatus = (unsigned char *)malloc((size_t)ntri + 1);
    memcpy(out->tstatus, S->ts, (size_t)ntri);
  }
  out->status = S->err;
  free(S->pts);
  free(S->ps);
  free(S->tri);
  free(S->nbr);
  free(S->t2s);
  free(S->ts);
  free(S->tmark);
  free(S->s2t.a);
  free(S->s2seg.a);
  free(S->enc.a);
  free(S->s2t_epoch);
  free(S->s2t_key);
  free(S->segs);
  free(S->emptyp.a);
  free(S->emptyt.a);
  free(S->l0.a);
  free(S->l1.a);
  free(S->l2.a);
  free(S->l3.a);
  free(S->l4.a);
  free(S->l5.a);
  return out->status;
}

void gqm_oracle_free(gqm_oracle_out *o) {
  free(o->pointlist);
  free(o->trianglelist);
  free(o->neighborlist);
  free(o->segmentlist);
  free(o->pstatus);
  free(o->tstatus);
  memset(o, 0, sizeof(*o));
}

double gqm_oracle_orient(const double *a, const double *b, const double *c) {
  P2 A = {a[0], a[1]}, B = {b[0], b[1]}, C = {c[0], c[1]};
  return orient_ref(A, B, C);
}
double gqm_oracle_incircle(const double *a, const double *b, const double *c, const double *d) {
  P2 A = {a[0], a[1]}, B = {b[0], b[1]}, C = {c[0], c[1]}, D = {d[0], d[1]};
  return incircle_pair(A, B, C, D);
}
double gqm_oracle_incircle_exact(const double *a, const double *b, const double *c, const double *d) {
  P2 A = {a[0], a[1]}, B = {b[0], b[1]}, C = {c[0], c[1]}, D = {d[0], d[1]};
  return incircle_expansion(A, B, C, D);
}
void gqm_oracle_circumcenter(const double *apex, const double *org, const double *dest, double offconstant,
                             int offcenter, double *o) {
  P2 A = {apex[0], apex[1]}, B = {org[0], org[1]}, C = {dest[0], dest[1]};
  P2 r = circumcenter(A, B, C, offconstant, offcenter);
  o[0] = r.x;
  o[1] = r.y;
}
