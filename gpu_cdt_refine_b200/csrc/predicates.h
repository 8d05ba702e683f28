// Orientation and incircle predicates shared by host and device code.
//
// Two families live here.
//
// 1. Reference-compatible ("ref") predicates.  The reference keeps its filter
//    constants in `__constant__ REAL constData[13]` (GPU_Refine/cudaCCW.h:41)
//    and never writes them, so every error bound and the Dekker splitter are
//    zero on the device.  The effective behaviour of its predicates is then:
//      cuda_fast / cuda_ccw  (cudaCCW.h:487-565): the plain FP64 determinant;
//      cuda_inCircle        (cudaCCW.h:668-708): the plain FP64 determinant
//                           when it is non-zero, else 0;
//      cuda_inCircle_exact  (cudaCCW.h:711-757): +-1 when the plain determinant
//                           is non-zero, else cuda_incircleexact (570-666)
//                           evaluated with splitter 0, which makes every
//                           Two_Product tail zero.
//    The functions below reproduce that arithmetic operation for operation.
//    They must be compiled without FMA contraction (nvcc -fmad=false,
//    gcc -ffp-contract=off) so that every product and sum is rounded on its
//    own, as in the reference built with -fmad=false.
//
// 2. Exact predicates (Shewchuk's adaptive-precision method: "Adaptive
//    Precision Floating-Point Arithmetic and Fast Robust Geometric Predicates",
//    1997).  A forward-error filter with the published bounds
//    (3+16e)e for orient2d and (10+96e)e for incircle, e = 2^-53, and an exact
//    expansion evaluation when the filter cannot decide.  Products use the
//    correctly rounded fma() for their error term.
#pragma once
#include <math.h>

#if defined(__CUDACC__)
#define GQM_HD __host__ __device__ __forceinline__
#else
#define GQM_HD static inline
#endif

typedef struct {
  double x, y;
} gqm_pt;

// ---------------------------------------------------------------------------
// Reference-compatible arithmetic
// ---------------------------------------------------------------------------

// Product-sum a * b + c of the reference's arithmetic.  The reference as its
// project builds it (nvcc's default -fmad=true) fuses some of its products into
// the add or subtract that consumes them; which ones was measured on its
// compiled kernels and predicates by comparing their outputs with every
// candidate evaluation.  With GQM_CONTRACTED set, the expressions of the
// reference's arithmetic use gqm_madd (one rounding, fma) exactly where that
// build fuses; without it gqm_madd rounds the product and the sum on their own
// (the reference built with -fmad=false).  Both variants are compiled without
// compiler contraction (nvcc -fmad=false, gcc -ffp-contract=off), so the
// arithmetic is the one written out here.
#ifndef GQM_CONTRACTED
#define GQM_CONTRACTED 0
#endif
GQM_HD double gqm_madd(double a, double b, double c) {
#if GQM_CONTRACTED
  return fma(a, b, c);
#else
  return a * b + c;
#endif
}

// cuda_fast / cuda_ccw with zero error bounds (cudaCCW.h:487-565).  Both
// products are rounded on their own in both builds of the reference (each is
// also used by the sign tests and the error bound).
GQM_HD double gqm_orient_ref(double ax, double ay, double bx, double by, double cx, double cy) {
  double detleft = (ax - cx) * (by - cy);
  double detright = (ay - cy) * (bx - cx);
  return detleft - detright;
}

// The plain incircle determinant of cuda_inCircle (cudaCCW.h:668-702).  The
// six cross products are rounded on their own in both builds of the reference
// (each is also used by the error bound's permanent); its contracted build
// fuses each lift's first square and the first and last terms of the sum.
GQM_HD double gqm_incircle_det_ref(double pax, double pay, double pbx, double pby, double pcx, double pcy,
                                   double pdx, double pdy) {
  double adx = pax - pdx, bdx = pbx - pdx, cdx = pcx - pdx;
  double ady = pay - pdy, bdy = pby - pdy, cdy = pcy - pdy;
  double bdxcdy = bdx * cdy;
  double cdxbdy = cdx * bdy;
  double alift = gqm_madd(adx, adx, ady * ady);
  double cdxady = cdx * ady;
  double adxcdy = adx * cdy;
  double blift = gqm_madd(bdx, bdx, bdy * bdy);
  double adxbdy = adx * bdy;
  double bdxady = bdx * ady;
  double clift = gqm_madd(cdx, cdx, cdy * cdy);
  return gqm_madd(clift, adxbdy - bdxady, gqm_madd(alift, bdxcdy - cdxbdy, blift * (cdxady - adxcdy)));
}

// --- expansion arithmetic with the reference's zero splitter ---------------
// Two_Sum / Two_Diff / Fast_Two_Sum are the standard error-free transforms.
// With splitter 0, Split(a) gives hi = a, lo = 0 and the product tail is +0.
GQM_HD void gqm__two_sum(double a, double b, double *x, double *y) {
  double s = a + b;
  double bv = s - a;
  double av = s - bv;
  double br = b - bv;
  double ar = a - av;
  *x = s;
  *y = ar + br;
}
GQM_HD void gqm__two_diff(double a, double b, double *x, double *y) {
  double s = a - b;
  double bv = a - s;
  double av = s + bv;
  double br = bv - b;
  double ar = a - av;
  *x = s;
  *y = ar + br;
}
GQM_HD void gqm__fast_two_sum(double a, double b, double *x, double *y) {
  double s = a + b;
  double bv = s - a;
  *x = s;
  *y = b - bv;
}
// Two_Product with a zero splitter and no FMA: the tail is always +0.0 for
// finite inputs (cudaCCW.h:119-131 with constData[0] == 0).
GQM_HD void gqm__two_product_z(double a, double b, double *x, double *y) {
  double p = a * b;
  double c = 0.0 * a;
  double abig = c - a;
  double ahi = c - abig;
  double alo = a - ahi;
  double cb = 0.0 * b;
  double bbig = cb - b;
  double bhi = cb - bbig;
  double blo = b - bhi;
  double err1 = p - (ahi * bhi);
  double err2 = err1 - (alo * bhi);
  double err3 = err2 - (ahi * blo);
  *x = p;
  *y = (alo * blo) - err3;
}
// Two_One_Diff then Two_Two_Diff (cudaCCW.h:166-176).
GQM_HD void gqm__two_two_diff(double a1, double a0, double b1, double b0, double *x3, double *x2, double *x1,
                              double *x0) {
  double i, j, z;
  double t1;
  // Two_One_Diff(a1, a0, b0, j, z, x0)
  gqm__two_diff(a0, b0, &i, x0);
  gqm__two_sum(a1, i, &j, &z);
  // Two_One_Diff(j, z, b1, x3, x2, x1)
  gqm__two_diff(z, b1, &i, x1);
  gqm__two_sum(j, i, x3, &t1);
  *x2 = t1;
}

// fast_expansion_sum_zeroelim (cudaCCW.h:196-258); e and f must not be read
// past their lengths, so the "next" element is fetched only when it exists.
GQM_HD int gqm__fast_expansion_sum_zeroelim(int elen, const double *e, int flen, const double *f, double *h) {
  double Q, Qnew, hh;
  int eindex = 0, findex = 0, hindex = 0;
  double enow = e[0];
  double fnow = f[0];
  if ((fnow > enow) == (fnow > -enow)) {
    Q = enow;
    ++eindex;
    enow = eindex < elen ? e[eindex] : 0.0;
  } else {
    Q = fnow;
    ++findex;
    fnow = findex < flen ? f[findex] : 0.0;
  }
  if ((eindex < elen) && (findex < flen)) {
    if ((fnow > enow) == (fnow > -enow)) {
      gqm__fast_two_sum(enow, Q, &Qnew, &hh);
      ++eindex;
      enow = eindex < elen ? e[eindex] : 0.0;
    } else {
      gqm__fast_two_sum(fnow, Q, &Qnew, &hh);
      ++findex;
      fnow = findex < flen ? f[findex] : 0.0;
    }
    Q = Qnew;
    if (hh != 0.0) h[hindex++] = hh;
    while ((eindex < elen) && (findex < flen)) {
      if ((fnow > enow) == (fnow > -enow)) {
        gqm__two_sum(Q, enow, &Qnew, &hh);
        ++eindex;
        enow = eindex < elen ? e[eindex] : 0.0;
      } else {
        gqm__two_sum(Q, fnow, &Qnew, &hh);
        ++findex;
        fnow = findex < flen ? f[findex] : 0.0;
      }
      Q = Qnew;
      if (hh != 0.0) h[hindex++] = hh;
    }
  }
  while (eindex < elen) {
    gqm__two_sum(Q, enow, &Qnew, &hh);
    ++eindex;
    enow = eindex < elen ? e[eindex] : 0.0;
    Q = Qnew;
    if (hh != 0.0) h[hindex++] = hh;
  }
  while (findex < flen) {
    gqm__two_sum(Q, fnow, &Qnew, &hh);
    ++findex;
    fnow = findex < flen ? f[findex] : 0.0;
    Q = Qnew;
    if (hh != 0.0) h[hindex++] = hh;
  }
  if ((Q != 0.0) || (hindex == 0)) h[hindex++] = Q;
  return hindex;
}

// scale_expansion_zeroelim (cudaCCW.h:276-313) with the zero splitter.
GQM_HD int gqm__scale_expansion_zeroelim_z(int elen, const double *e, double b, double *h) {
  double Q, sum, hh, product1, product0;
  int hindex = 0;
  gqm__two_product_z(e[0], b, &Q, &hh);
  if (hh != 0) h[hindex++] = hh;
  for (int eindex = 1; eindex < elen; eindex++) {
    gqm__two_product_z(e[eindex], b, &product1, &product0);
    gqm__two_sum(Q, product0, &sum, &hh);
    if (hh != 0) h[hindex++] = hh;
    gqm__fast_two_sum(product1, sum, &Q, &hh);
    if (hh != 0) h[hindex++] = hh;
  }
  if ((Q != 0.0) || (hindex == 0)) h[hindex++] = Q;
  return hindex;
}

// cuda_incircleexact (cudaCCW.h:570-666) evaluated with the zero splitter.
// Reached by the reference only when the plain determinant is exactly zero.
GQM_HD double gqm_incircle_zero_fallback_ref(double pax, double pay, double pbx, double pby, double pcx, double pcy,
                                             double pdx, double pdy) {
  double x1, x0, y1, y0;
  double ab[4], bc[4], cd[4], da[4], ac[4], bd[4];
  double temp8[8];
  double abc[12], bcd[12], cda[12], dab[12];
  double det24x[24], det24y[24], det48x[48], det48y[48];
  double adet[96], bdet[96], cdet[96], ddet[96];
  double abdet[192], cddet[192];
  double deter[384];
  int templen, abclen, bcdlen, cdalen, dablen, xlen, ylen, alen, blen, clen, dlen, ablen, cdlen, deterlen;

  gqm__two_product_z(pax, pby, &x1, &x0);
  gqm__two_product_z(pbx, pay, &y1, &y0);
  gqm__two_two_diff(x1, x0, y1, y0, &ab[3], &ab[2], &ab[1], &ab[0]);
  gqm__two_product_z(pbx, pcy, &x1, &x0);
  gqm__two_product_z(pcx, pby, &y1, &y0);
  gqm__two_two_diff(x1, x0, y1, y0, &bc[3], &bc[2], &bc[1], &bc[0]);
  gqm__two_product_z(pcx, pdy, &x1, &x0);
  gqm__two_product_z(pdx, pcy, &y1, &y0);
  gqm__two_two_diff(x1, x0, y1, y0, &cd[3], &cd[2], &cd[1], &cd[0]);
  gqm__two_product_z(pdx, pay, &x1, &x0);
  gqm__two_product_z(pax, pdy, &y1, &y0);
  gqm__two_two_diff(x1, x0, y1, y0, &da[3], &da[2], &da[1], &da[0]);
  gqm__two_product_z(pax, pcy, &x1, &x0);
  gqm__two_product_z(pcx, pay, &y1, &y0);
  gqm__two_two_diff(x1, x0, y1, y0, &ac[3], &ac[2], &ac[1], &ac[0]);
  gqm__two_product_z(pbx, pdy, &x1, &x0);
  gqm__two_product_z(pdx, pby, &y1, &y0);
  gqm__two_two_diff(x1, x0, y1, y0, &bd[3], &bd[2], &bd[1], &bd[0]);

  templen = gqm__fast_expansion_sum_zeroelim(4, cd, 4, da, temp8);
  cdalen = gqm__fast_expansion_sum_zeroelim(templen, temp8, 4, ac, cda);
  templen = gqm__fast_expansion_sum_zeroelim(4, da, 4, ab, temp8);
  dablen = gqm__fast_expansion_sum_zeroelim(templen, temp8, 4, bd, dab);
  for (int i = 0; i < 4; i++) {
    bd[i] = -bd[i];
    ac[i] = -ac[i];
  }
  templen = gqm__fast_expansion_sum_zeroelim(4, ab, 4, bc, temp8);
  abclen = gqm__fast_expansion_sum_zeroelim(templen, temp8, 4, ac, abc);
  templen = gqm__fast_expansion_sum_zeroelim(4, bc, 4, cd, temp8);
  bcdlen = gqm__fast_expansion_sum_zeroelim(templen, temp8, 4, bd, bcd);

  xlen = gqm__scale_expansion_zeroelim_z(bcdlen, bcd, pax, det24x);
  xlen = gqm__scale_expansion_zeroelim_z(xlen, det24x, pax, det48x);
  ylen = gqm__scale_expansion_zeroelim_z(bcdlen, bcd, pay, det24y);
  ylen = gqm__scale_expansion_zeroelim_z(ylen, det24y, pay, det48y);
  alen = gqm__fast_expansion_sum_zeroelim(xlen, det48x, ylen, det48y, adet);

  xlen = gqm__scale_expansion_zeroelim_z(cdalen, cda, pbx, det24x);
  xlen = gqm__scale_expansion_zeroelim_z(xlen, det24x, -pbx, det48x);
  ylen = gqm__scale_expansion_zeroelim_z(cdalen, cda, pby, det24y);
  ylen = gqm__scale_expansion_zeroelim_z(ylen, det24y, -pby, det48y);
  blen = gqm__fast_expansion_sum_zeroelim(xlen, det48x, ylen, det48y, bdet);

  xlen = gqm__scale_expansion_zeroelim_z(dablen, dab, pcx, det24x);
  xlen = gqm__scale_expansion_zeroelim_z(xlen, det24x, pcx, det48x);
  ylen = gqm__scale_expansion_zeroelim_z(dablen, dab, pcy, det24y);
  ylen = gqm__scale_expansion_zeroelim_z(ylen, det24y, pcy, det48y);
  clen = gqm__fast_expansion_sum_zeroelim(xlen, det48x, ylen, det48y, cdet);

  xlen = gqm__scale_expansion_zeroelim_z(abclen, abc, pdx, det24x);
  xlen = gqm__scale_expansion_zeroelim_z(xlen, det24x, -pdx, det48x);
  ylen = gqm__scale_expansion_zeroelim_z(abclen, abc, pdy, det24y);
  ylen = gqm__scale_expansion_zeroelim_z(ylen, det24y, -pdy, det48y);
  dlen = gqm__fast_expansion_sum_zeroelim(xlen, det48x, ylen, det48y, ddet);

  ablen = gqm__fast_expansion_sum_zeroelim(alen, adet, blen, bdet, abdet);
  cdlen = gqm__fast_expansion_sum_zeroelim(clen, cdet, dlen, ddet, cddet);
  deterlen = gqm__fast_expansion_sum_zeroelim(ablen, abdet, cdlen, cddet, deter);
  return deter[deterlen - 1];
}

// ---------------------------------------------------------------------------
// Exact predicates (robust mode, CDT construction and output certificate)
// ---------------------------------------------------------------------------
#define GQM_EPS 1.1102230246251565e-16 /* 2^-53 */

GQM_HD void gqm__two_product_x(double a, double b, double *x, double *y) {
  double p = a * b;
  *x = p;
  *y = fma(a, b, -p);
}
// Exact a*b - c*d as a 4-component expansion (Two_Two_Diff of two products).
GQM_HD void gqm__cross_x(double a, double b, double c, double d, double *r) {
  double x1, x0, y1, y0, i, j, z, t;
  gqm__two_product_x(a, b, &x1, &x0);
  gqm__two_product_x(c, d, &y1, &y0);
  gqm__two_diff(x0, y0, &i, &r[0]);
  gqm__two_sum(x1, i, &j, &z);
  gqm__two_diff(z, y1, &i, &r[1]);
  gqm__two_sum(j, i, &r[3], &t);
  r[2] = t;
}
GQM_HD int gqm__scale_expansion_x(int elen, const double *e, double b, double *h) {
  double Q, sum, hh, product1, product0;
  int hindex = 0;
  gqm__two_product_x(e[0], b, &Q, &hh);
  if (hh != 0) h[hindex++] = hh;
  for (int eindex = 1; eindex < elen; eindex++) {
    gqm__two_product_x(e[eindex], b, &product1, &product0);
    gqm__two_sum(Q, product0, &sum, &hh);
    if (hh != 0) h[hindex++] = hh;
    gqm__fast_two_sum(product1, sum, &Q, &hh);
    if (hh != 0) h[hindex++] = hh;
  }
  if ((Q != 0.0) || (hindex == 0)) h[hindex++] = Q;
  return hindex;
}

// Exact orient2d: positive if a, b, c are counterclockwise.
GQM_HD double gqm_orient_exact(double ax, double ay, double bx, double by, double cx, double cy) {
  double detleft = (ax - cx) * (by - cy);
  double detright = (ay - cy) * (bx - cx);
  double det = detleft - detright;
  double detsum;
  if (detleft > 0.0) {
    if (detright <= 0.0) return det;
    detsum = detleft + detright;
  } else if (detleft < 0.0) {
    if (detright >= 0.0) return det;
    detsum = -detleft - detright;
  } else {
    return det;
  }
  double errbound = (3.0 + 16.0 * GQM_EPS) * GQM_EPS * detsum;
  if ((det >= errbound) || (-det >= errbound)) return det;
  // exact: a.x*b.y - a.x*c.y + b.x*c.y - b.x*a.y + c.x*a.y - c.x*b.y
  double t1[4], t2[4], t3[4], v[8], w[12];
  gqm__cross_x(ax, by, ax, cy, t1);
  gqm__cross_x(bx, cy, bx, ay, t2);
  gqm__cross_x(cx, ay, cx, by, t3);
  int vl = gqm__fast_expansion_sum_zeroelim(4, t1, 4, t2, v);
  int wl = gqm__fast_expansion_sum_zeroelim(vl, v, 4, t3, w);
  return w[wl - 1];
}

// Exact incircle: positive if d lies inside the circle through a, b, c
// (a, b, c counterclockwise).
GQM_HD double gqm_incircle_exact(double pax, double pay, double pbx, double pby, double pcx, double pcy, double pdx,
                                 double pdy) {
  double adx = pax - pdx, bdx = pbx - pdx, cdx = pcx - pdx;
  double ady = pay - pdy, bdy = pby - pdy, cdy = pcy - pdy;
  double bdxcdy = bdx * cdy, cdxbdy = cdx * bdy;
  double alift = adx * adx + ady * ady;
  double cdxady = cdx * ady, adxcdy = adx * cdy;
  double blift = bdx * bdx + bdy * bdy;
  double adxbdy = adx * bdy, bdxady = bdx * ady;
  double clift = cdx * cdx + cdy * cdy;
  double det = alift * (bdxcdy - cdxbdy) + blift * (cdxady - adxcdy) + clift * (adxbdy - bdxady);
  double permanent = (fabs(bdxcdy) + fabs(cdxbdy)) * alift + (fabs(cdxady) + fabs(adxcdy)) * blift +
                     (fabs(adxbdy) + fabs(bdxady)) * clift;
  double errbound = (10.0 + 96.0 * GQM_EPS) * GQM_EPS * permanent;
  if ((det > errbound) || (-det > errbound)) return det;

  // Exact evaluation of the 4x4 lifted determinant (Shewchuk's incircleexact
  // decomposition into 2x2 minors of the absolute coordinates).
  double ab[4], bc[4], cd[4], da[4], ac[4], bd[4];
  double temp8[8], abc[12], bcd[12], cda[12], dab[12];
  double det24x[24], det24y[24], det48x[48], det48y[48];
  double adet[96], bdet[96], cdet[96], ddet[96];
  double abdet[192], cddet[192], deter[384];
  gqm__cross_x(pax, pby, pbx, pay, ab);
  gqm__cross_x(pbx, pcy, pcx, pby, bc);
  gqm__cross_x(pcx, pdy, pdx, pcy, cd);
  gqm__cross_x(pdx, pay, pax, pdy, da);
  gqm__cross_x(pax, pcy, pcx, pay, ac);
  gqm__cross_x(pbx, pdy, pdx, pby, bd);
  int tl = gqm__fast_expansion_sum_zeroelim(4, cd, 4, da, temp8);
  int cdal = gqm__fast_expansion_sum_zeroelim(tl, temp8, 4, ac, cda);
  tl = gqm__fast_expansion_sum_zeroelim(4, da, 4, ab, temp8);
  int dabl = gqm__fast_expansion_sum_zeroelim(tl, temp8, 4, bd, dab);
  for (int i = 0; i < 4; i++) {
    bd[i] = -bd[i];
    ac[i] = -ac[i];
  }
  tl = gqm__fast_expansion_sum_zeroelim(4, ab, 4, bc, temp8);
  int abcl = gqm__fast_expansion_sum_zeroelim(tl, temp8, 4, ac, abc);
  tl = gqm__fast_expansion_sum_zeroelim(4, bc, 4, cd, temp8);
  int bcdl = gqm__fast_expansion_sum_zeroelim(tl, temp8, 4, bd, bcd);
  int xl, yl;
  xl = gqm__scale_expansion_x(bcdl, bcd, pax, det24x);
  xl = gqm__scale_expansion_x(xl, det24x, pax, det48x);
  yl = gqm__scale_expansion_x(bcdl, bcd, pay, det24y);
  yl = gqm__scale_expansion_x(yl, det24y, pay, det48y);
  int al = gqm__fast_expansion_sum_zeroelim(xl, det48x, yl, det48y, adet);
  xl = gqm__scale_expansion_x(cdal, cda, pbx, det24x);
  xl = gqm__scale_expansion_x(xl, det24x, -pbx, det48x);
  yl = gqm__scale_expansion_x(cdal, cda, pby, det24y);
  yl = gqm__scale_expansion_x(yl, det24y, -pby, det48y);
  int bl = gqm__fast_expansion_sum_zeroelim(xl, det48x, yl, det48y, bdet);
  xl = gqm__scale_expansion_x(dabl, dab, pcx, det24x);
  xl = gqm__scale_expansion_x(xl, det24x, pcx, det48x);
  yl = gqm__scale_expansion_x(dabl, dab, pcy, det24y);
  yl = gqm__scale_expansion_x(yl, det24y, pcy, det48y);
  int cl = gqm__fast_expansion_sum_zeroelim(xl, det48x, yl, det48y, cdet);
  xl = gqm__scale_expansion_x(abcl, abc, pdx, det24x);
  xl = gqm__scale_expansion_x(xl, det24x, -pdx, det48x);
  yl = gqm__scale_expansion_x(abcl, abc, pdy, det24y);
  yl = gqm__scale_expansion_x(yl, det24y, -pdy, det48y);
  int dl = gqm__fast_expansion_sum_zeroelim(xl, det48x, yl, det48y, ddet);
  int abl = gqm__fast_expansion_sum_zeroelim(al, adet, bl, bdet, abdet);
  int cdl2 = gqm__fast_expansion_sum_zeroelim(cl, cdet, dl, ddet, cddet);
  int dtl = gqm__fast_expansion_sum_zeroelim(abl, abdet, cdl2, cddet, deter);
  return deter[dtl - 1];
}
