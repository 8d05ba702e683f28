/* Candidate evaluations of the reference's floating-point expressions, one per
 * way nvcc's contraction can fuse a product into the add or subtract that
 * consumes it: unfused (v 0), first product fused (fma(a, b, c*d), v 1),
 * second product fused (fma(c, d, a*b), v 2).  Compiled with
 * -ffp-contract=off, so each candidate is exactly the arithmetic it writes.
 * analyze.py compares them bit for bit with the outputs of the reference's
 * own compiled predicates and kernels (probe_predicates.cu, probe_kernels.cu).
 * Test infrastructure: it decides which products the oracle's and the
 * contracted library's gqm_madd / madd sites fuse. */
#include <math.h>

/* cuda_ccw / cuda_fast (GPU_Refine/cudaCCW.h:487-565) */
double ccw_v(const double *a, const double *b, const double *c, int v) {
  double l1 = a[0] - c[0], l2 = b[1] - c[1], r1 = a[1] - c[1], r2 = b[0] - c[0];
  double L = l1 * l2, R = r1 * r2;
  if (v == 0) return L - R;
  if (v == 1) return fma(l1, l2, -R);
  return fma(-r1, r2, L);
}
/* cuda_inCircle (cudaCCW.h:668-708).  v: bits 0-1 the three cross differences,
   bits 2-3 the lifts, bits 4-6 the order of the fused terms of the sum */
double inc_v(const double *pa, const double *pb, const double *pc, const double *pd, int v) {
  double adx = pa[0] - pd[0], bdx = pb[0] - pd[0], cdx = pc[0] - pd[0];
  double ady = pa[1] - pd[1], bdy = pb[1] - pd[1], cdy = pc[1] - pd[1];
  double bdxcdy = bdx * cdy, cdxbdy = cdx * bdy, cdxady = cdx * ady, adxcdy = adx * cdy, adxbdy = adx * bdy,
         bdxady = bdx * ady;
  double d1, d2, d3;
  int cv = v & 3;
  if (cv == 0) { d1 = bdxcdy - cdxbdy; d2 = cdxady - adxcdy; d3 = adxbdy - bdxady; }
  else if (cv == 1) { d1 = fma(bdx, cdy, -cdxbdy); d2 = fma(cdx, ady, -adxcdy); d3 = fma(adx, bdy, -bdxady); }
  else { d1 = fma(-cdx, bdy, bdxcdy); d2 = fma(-adx, cdy, cdxady); d3 = fma(-bdx, ady, adxbdy); }
  double al, bl, cl;
  int lv = (v >> 2) & 3;
  if (lv == 0) { al = adx * adx + ady * ady; bl = bdx * bdx + bdy * bdy; cl = cdx * cdx + cdy * cdy; }
  else if (lv == 1) { al = fma(adx, adx, ady * ady); bl = fma(bdx, bdx, bdy * bdy); cl = fma(cdx, cdx, cdy * cdy); }
  else { al = fma(ady, ady, adx * adx); bl = fma(bdy, bdy, bdx * bdx); cl = fma(cdy, cdy, cdx * cdx); }
  int sv = (v >> 4) & 7;
  double t1 = al * d1, t2 = bl * d2, t3 = cl * d3;
  switch (sv) {
    case 0: return (t1 + t2) + t3;
    case 1: return fma(cl, d3, fma(al, d1, t2));
    case 2: return fma(cl, d3, fma(bl, d2, t1));
    case 3: return fma(cl, d3, t1 + t2);
    case 4: return fma(al, d1, t2) + t3;
    default: return fma(bl, d2, t1) + t3;
  }
}
typedef struct { double x, y; } P;
static double sq(double dx, double dy, int v) {
  if (v == 0) { double a = dx * dx, b = dy * dy; return a + b; }
  if (v == 1) { double b = dy * dy; return fma(dx, dx, b); }
  double a = dx * dx; return fma(dy, dy, a);
}
/* a*b - c*d */
static double dd(double a, double b, double c, double d, int v) {
  if (v == 0) { double x = a * b, y = c * d; return x - y; }
  if (v == 1) { double y = c * d; return fma(a, b, -y); }
  double x = a * b; return fma(-c, d, x);
}
/* a*b + c*d */
static double ds(double a, double b, double c, double d, int v) {
  if (v == 0) { double x = a * b, y = c * d; return x + y; }
  if (v == 1) { double y = c * d; return fma(a, b, y); }
  double x = a * b; return fma(c, d, x);
}
/* computeCircumcenter, refine.cu:3780-3868; opt: [dist, tmp, numx, numy, offx, offy, cmp] */
void cc_cand(const double *pa, const double *po, const double *pd, double offc, int offcenter, const int *o,
             double *out) {
  P vApex = {pa[0], pa[1]}, vOrg = {po[0], po[1]}, vDest = {pd[0], pd[1]};
  double xdo = vDest.x - vOrg.x, ydo = vDest.y - vOrg.y, xao = vApex.x - vOrg.x, yao = vApex.y - vOrg.y;
  double dodist = sq(xdo, ydo, o[0]), aodist = sq(xao, yao, o[0]);
  double dadist = sq(vDest.x - vApex.x, vDest.y - vApex.y, o[0]);
  double tmp = dd(xdo, yao, xao, ydo, o[1]);
  double den = 0.5 / tmp;
  double dx = dd(yao, dodist, ydo, aodist, o[2]) * den;
  double dy = dd(xdo, aodist, xao, dodist, o[3]) * den;
  if (offcenter && offc > 0.0) {
    double dxoff, dyoff;
    if (dodist < aodist && dodist < dadist) {
      dxoff = o[4] ? fma(-offc, ydo, 0.5 * xdo) : 0.5 * xdo - offc * ydo;
      dyoff = o[5] ? fma(offc, xdo, 0.5 * ydo) : 0.5 * ydo + offc * xdo;
      if (sq(dxoff, dyoff, o[6]) < sq(dx, dy, o[6])) { dx = dxoff; dy = dyoff; }
    } else if (aodist < dadist) {
      dxoff = o[5] ? fma(offc, yao, 0.5 * xao) : 0.5 * xao + offc * yao;
      dyoff = o[4] ? fma(-offc, xao, 0.5 * yao) : 0.5 * yao - offc * xao;
      if (sq(dxoff, dyoff, o[6]) < sq(dx, dy, o[6])) { dx = dxoff; dy = dyoff; }
    } else {
      double ex = vApex.x - vDest.x, ey = vApex.y - vDest.y;
      dxoff = o[4] ? fma(-offc, ey, 0.5 * ex) : 0.5 * ex - offc * ey;
      dyoff = o[5] ? fma(offc, ex, 0.5 * ey) : 0.5 * ey + offc * ex;
      if (sq(dxoff, dyoff, o[6]) < sq(dx - xdo, dy - ydo, o[6])) { dx = xdo + dxoff; dy = ydo + dyoff; }
    }
  }
  out[0] = vOrg.x + dx;
  out[1] = vOrg.y + dy;
}
/* kernelComputeSmallestAngle + bad test (refine.cu:317-374, 418-420); o: [len, dot] */
int bad_cand(const double *pa, const double *po, const double *pd, double gc2, const int *o) {
  double dxod = po[0] - pd[0], dyod = po[1] - pd[1], dxda = pd[0] - pa[0], dyda = pd[1] - pa[1];
  double dxao = pa[0] - po[0], dyao = pa[1] - po[1];
  double lo = sq(dxod, dyod, o[0]), ld = sq(dxda, dyda, o[0]), la = sq(dxao, dyao, o[0]);
  double ang, s;
  if (lo < ld && lo < la) { s = lo; ang = ds(dxda, dxao, dyda, dyao, o[1]); }
  else if (ld < lo && ld < la) { s = ld; ang = ds(dxod, dxao, dyod, dyao, o[1]); }
  else { s = la; ang = ds(dxod, dxda, dyod, dyda, o[1]); }
  double c2 = ang * ang * s / (lo * ld * la);
  return c2 > gc2;
}
/* checkseg4encroach (refine.cu:115-139); o: [dot, len] */
int enc_cand(const double *o_, const double *d_, const double *a_, double gcs, int mode, const int *o) {
  double dot = ds(o_[0] - a_[0], d_[0] - a_[0], o_[1] - a_[1], d_[1] - a_[1], o[0]);
  if (dot < 0.0) {
    if (mode) return 1;
    double k = 2.0 * gcs - 1.0;
    double l1 = sq(o_[0] - a_[0], o_[1] - a_[1], o[1]), l2 = sq(d_[0] - a_[0], d_[1] - a_[1], o[1]);
    if (dot * dot >= k * k * l1 * l2) return 1;
  }
  return 0;
}
/* per-length and per-branch options: o = [lo, ld, la, dot0, dot1, dot2] */
static int bad_cand2(const double *pa, const double *po, const double *pd, double gc2, const int *o) {
  double dxod = po[0] - pd[0], dyod = po[1] - pd[1], dxda = pd[0] - pa[0], dyda = pd[1] - pa[1];
  double dxao = pa[0] - po[0], dyao = pa[1] - po[1];
  double lo = sq(dxod, dyod, o[0]), ld = sq(dxda, dyda, o[1]), la = sq(dxao, dyao, o[2]);
  double ang, s;
  if (lo < ld && lo < la) { s = lo; ang = ds(dxda, dxao, dyda, dyao, o[3]); }
  else if (ld < lo && ld < la) { s = ld; ang = ds(dxod, dxao, dyod, dyao, o[4]); }
  else { s = la; ang = ds(dxod, dxda, dyod, dyda, o[5]); }
  double c2 = ang * ang * s / (lo * ld * la);
  return c2 > gc2;
}
void bad_search(const double *P, const unsigned char *bad, int n, double gc2, int *score /* 729 */) {
  int o[6];
  for (int k = 0; k < 729; ++k) {
    int t = k;
    for (int j = 0; j < 6; ++j) { o[j] = t % 3; t /= 3; }
    int ok = 0;
    for (int i = 0; i < n; ++i) ok += bad_cand2(P + 6 * i, P + 6 * i + 2, P + 6 * i + 4, gc2, o) == bad[i];
    score[k] = ok;
  }
}
/* offcenter with per-branch options: o = [b0x, b0y, b1x, b1y, b2x, b2y, cmpL, cmpR] (x: the "-" term, y: the "+") */
static void off_cand(const double *pa, const double *po, const double *pd, double offc, const int *o, double *out) {
  P vApex = {pa[0], pa[1]}, vOrg = {po[0], po[1]}, vDest = {pd[0], pd[1]};
  double xdo = vDest.x - vOrg.x, ydo = vDest.y - vOrg.y, xao = vApex.x - vOrg.x, yao = vApex.y - vOrg.y;
  double dodist = sq(xdo, ydo, 1), aodist = sq(xao, yao, 1);
  double dadist = sq(vDest.x - vApex.x, vDest.y - vApex.y, 1);
  double tmp = dd(xdo, yao, xao, ydo, 0);
  double den = 0.5 / tmp;
  double dx = dd(yao, dodist, ydo, aodist, 1) * den;
  double dy = dd(xdo, aodist, xao, dodist, 1) * den;
  double dxoff, dyoff;
  if (dodist < aodist && dodist < dadist) {
    dxoff = o[0] ? fma(-offc, ydo, 0.5 * xdo) : 0.5 * xdo - offc * ydo;
    dyoff = o[1] ? fma(offc, xdo, 0.5 * ydo) : 0.5 * ydo + offc * xdo;
    if (sq(dxoff, dyoff, o[6]) < sq(dx, dy, o[7])) { dx = dxoff; dy = dyoff; }
  } else if (aodist < dadist) {
    dxoff = o[3] ? fma(offc, yao, 0.5 * xao) : 0.5 * xao + offc * yao;
    dyoff = o[2] ? fma(-offc, xao, 0.5 * yao) : 0.5 * yao - offc * xao;
    if (sq(dxoff, dyoff, o[6]) < sq(dx, dy, o[7])) { dx = dxoff; dy = dyoff; }
  } else {
    double ex = vApex.x - vDest.x, ey = vApex.y - vDest.y;
    dxoff = o[4] ? fma(-offc, ey, 0.5 * ex) : 0.5 * ex - offc * ey;
    dyoff = o[5] ? fma(offc, ex, 0.5 * ey) : 0.5 * ey + offc * ex;
    if (sq(dxoff, dyoff, o[6]) < sq(dx - xdo, dy - ydo, o[7])) { dx = xdo + dxoff; dy = ydo + dyoff; }
  }
  out[0] = vOrg.x + dx;
  out[1] = vOrg.y + dy;
}
void off_search(const double *P3, const double *cc, int n, double offc, int *score /* 576 */, int *branch_count) {
  int o[8];
  for (int k = 0; k < 576; ++k) {
    int t = k;
    for (int j = 0; j < 6; ++j) { o[j] = t % 2; t /= 2; }
    o[6] = t % 3; t /= 3; o[7] = t % 3;
    int ok = 0;
    double out[2];
    for (int i = 0; i < n; ++i) {
      off_cand(P3 + 6 * i, P3 + 6 * i + 2, P3 + 6 * i + 4, offc, o, out);
      ok += out[0] == cc[2 * i] && out[1] == cc[2 * i + 1];
    }
    score[k] = ok;
  }
}
