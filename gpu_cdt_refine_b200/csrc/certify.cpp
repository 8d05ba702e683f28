// Independent certificate for a refined constrained Delaunay triangulation.
//
// The reference only has ad-hoc, disabled checks (GPU_Refine/main.cpp:79-380:
// neighbour symmetry, input points preserved, minimum angle; the incircle
// check is commented out).  This certificate makes them exact:
//   1. every triangle is counterclockwise (exact orient2d > 0) and the
//      neighbour relation is symmetric; boundary edges are segments;
//   2. constrained Delaunay: across every edge that is not a segment, the
//      opposite vertex is not strictly inside the circumcircle (exact
//      incircle <= 0);
//   3. every input segment is the union of output segments: walking from one
//      endpoint along output segments, always moving forward along the
//      segment, reaches the other endpoint.  Split points are rounded FP64
//      values (the reference projects them back onto the line,
//      GPU_Refine/refine.cu:2712-2725, but cannot make them exactly
//      collinear), so the largest distance of a split point from its input
//      segment, relative to the segment length, is reported as well;
//   4. the input points are preserved at their indices;
//   5. quality, decided exactly: an angle at vertex o of a triangle (o, p, q)
//      is below theta iff dot(p - o, q - o) > 0 and
//      dot^2 > c2 * |p - o|^2 * |q - o|^2, with c2 the FP64 value of
//      cos^2(theta) that the refiner's bad-triangle test uses
//      (GPU_Refine/refine.cu:418-419; by default the host's cos(), or the
//      value the device computed when the caller passes it).  Both sides are
//      polynomials of degree 4 in the coordinates, evaluated with an FP64
//      filter and, when the filter cannot decide, exact expansion arithmetic
//      (Shewchuk's two-sum / scale-expansion, the same building blocks as the
//      exact predicates).  The only inexactness is in c2 itself: a relative
//      error of a few units in 2^-53 in cos^2(theta), i.e. the certified bound
//      is theta to within about 1e-14 degrees;
//   6. every triangle below theta is checked against the reference's one
//      exemption (GPU_Refine/refine.cu:426-493): its shortest edge is not a
//      segment, joins two split points of input segments, those two input
//      segments share an endpoint, and the endpoint is at nearly the same
//      distance from both split points (0.999 d2 < d1 < 1.001 d2, decided
//      exactly for the FP64 constants 0.999 and 1.001).  Split points and
//      their input segments come from the segment walk of check 3.  A
//      triangle below theta that the exemption does not cover is a quality
//      violation and fails the certificate, unless rule 7 covers it;
//   7. the reference's smallest-angle routine (GPU_Refine/refine.cu:317-374)
//      picks the shortest edge with strict comparisons of FP64 squared
//      lengths, so when the two shortest edges compare equal it falls through
//      to edge 2 and measures the angle opposite edge 2 instead of the
//      smallest one.  An isosceles triangle whose equal legs are its two
//      shortest edges (an off-center on the bisector of a short edge makes
//      them) can then pass the reference's bad test with an apex angle below
//      theta.  A triangle below theta is "tie_passed" when the reference's
//      FP64 test, evaluated as the reference writes it (every operation
//      rounded on its own), takes such a tie and judges the triangle good
//      (refine.cu:418-419);
//   8. minimum angle statistics (degrees, FP64 atan2 of exact-enough
//      cross/dot products).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "predicates.h"

extern "C" {

struct gqm_certificate {
  long long not_ccw, bad_neighbors, open_boundary, non_delaunay, segments_missing, input_points_moved;
  long long triangles_below_theta, euler_defect;
  double min_angle_deg, theta, max_segment_deviation;
  long long exempted;            /* triangles below theta that the reference's exemption covers */
  long long quality_violations;  /* triangles below theta that it does not */
  double goodcos2;               /* the cos^2(theta) the quality test used */
  long long tie_passed;          /* triangles below theta that the reference's FP64 test passes on a length tie */
};

}  // extern "C"

namespace {

// Exact arithmetic on expansions (nonoverlapping, increasing magnitude).
typedef std::vector<double> Exp;

Exp ex_diff(double a, double b) {
  double x, y;
  gqm__two_diff(a, b, &x, &y);
  return y != 0.0 ? Exp{y, x} : Exp{x};
}
Exp ex_add(const Exp &a, const Exp &b) {
  Exp h(a.size() + b.size());
  h.resize((size_t)gqm__fast_expansion_sum_zeroelim((int)a.size(), a.data(), (int)b.size(), b.data(), h.data()));
  return h;
}
Exp ex_scale(const Exp &a, double b) {
  Exp h(2 * a.size());
  h.resize((size_t)gqm__scale_expansion_x((int)a.size(), a.data(), b, h.data()));
  return h;
}
Exp ex_mul(const Exp &a, const Exp &b) {
  Exp acc{0.0};
  for (double t : b) acc = ex_add(acc, ex_scale(a, t));
  return acc;
}
Exp ex_neg(Exp a) {
  for (double &t : a) t = -t;
  return a;
}
int ex_sign(const Exp &a) {
  for (size_t i = a.size(); i-- > 0;)
    if (a[i] != 0.0) return a[i] > 0 ? 1 : -1;
  return 0;
}

// sign of dot(p - o, q - o)^2 - c2 |p - o|^2 |q - o|^2 when dot > 0, else -1:
// +1 means the angle at o is below theta
int angle_below(const gqm_pt &o, const gqm_pt &p, const gqm_pt &q, double c2) {
  const double ux = p.x - o.x, uy = p.y - o.y, wx = q.x - o.x, wy = q.y - o.y;
  const double dot = ux * wx + uy * wy, lu = ux * ux + uy * uy, lw = wx * wx + wy * wy;
  const double lhs = dot * dot, rhs = c2 * lu * lw;
  // FP64 filter: each side carries a relative error of at most ~12 units in
  // 2^-53 (differences, products and one sum); 1e-12 leaves a wide margin
  if (dot < 0 && fabs(dot) > 1e-12 * (fabs(ux * wx) + fabs(uy * wy))) return -1;
  if (fabs(lhs - rhs) > 1e-12 * (lhs + rhs)) {
    if (dot > 1e-12 * (fabs(ux * wx) + fabs(uy * wy))) return lhs > rhs ? 1 : -1;
  }
  const Exp eux = ex_diff(p.x, o.x), euy = ex_diff(p.y, o.y), ewx = ex_diff(q.x, o.x), ewy = ex_diff(q.y, o.y);
  const Exp edot = ex_add(ex_mul(eux, ewx), ex_mul(euy, ewy));
  if (ex_sign(edot) <= 0) return -1;
  const Exp elu = ex_add(ex_mul(eux, eux), ex_mul(euy, euy)), elw = ex_add(ex_mul(ewx, ewx), ex_mul(ewy, ewy));
  const Exp d = ex_add(ex_mul(edot, edot), ex_neg(ex_scale(ex_mul(elu, elw), c2)));
  return ex_sign(d);
}
// The reference's bad-triangle test in FP64 (GPU_Refine/refine.cu:317-374,
// 418-419) for a triangle (apex, org, dest), every operation rounded on its
// own (this file is compiled with -ffp-contract=off).  Returns true when the
// two shortest edges' squared lengths compare equal, so that the strict
// comparisons fall through to edge 2, and the cos^2 then measured is at most
// goodcos2 (the triangle passes as good).
bool reference_tie_passes(const gqm_pt &apex, const gqm_pt &org, const gqm_pt &dest, double goodcos2) {
  double dxod = org.x - dest.x, dyod = org.y - dest.y;
  double dxda = dest.x - apex.x, dyda = dest.y - apex.y;
  double dxao = apex.x - org.x, dyao = apex.y - org.y;
  double dxod2 = dxod * dxod, dyod2 = dyod * dyod, dxda2 = dxda * dxda, dyda2 = dyda * dyda;
  double dxao2 = dxao * dxao, dyao2 = dyao * dyao;
  const double len_org = dxod2 + dyod2, len_dest = dxda2 + dyda2, len_apex = dxao2 + dyao2;
  if (len_org < len_dest && len_org < len_apex) return false;
  if (len_dest < len_org && len_dest < len_apex) return false;
  // edge 2 is taken; a tie only if edge 2 is not itself strictly the shortest
  if (len_apex < len_org && len_apex < len_dest) return false;
  const double dot = dxod * dxda + dyod * dyda;
  const double cos2 = dot * dot * len_apex / (len_org * len_dest * len_apex);
  return cos2 <= goodcos2;
}
// exact squared distance of a and b
Exp ex_dist2(const gqm_pt &a, const gqm_pt &b) {
  const Exp dx = ex_diff(a.x, b.x), dy = ex_diff(a.y, b.y);
  return ex_add(ex_mul(dx, dx), ex_mul(dy, dy));
}

}  // namespace

extern "C" {

static inline uint64_t ekey(int a, int b) {
  uint32_t lo = (uint32_t)std::min(a, b), hi = (uint32_t)std::max(a, b);
  return ((uint64_t)hi << 32) | lo;
}

int gqm_certify(int np, const double *pts, int nt, const int *tri, const int *nbr, int ns, const int *segs,
                int nin, const double *in_pts, int nin_seg, const int *in_segs, double theta, double goodcos2,
                gqm_certificate *c) {
  memset(c, 0, sizeof(*c));
  c->theta = theta;
  if (!(goodcos2 > 0.0)) {
    const double cg = cos(theta * 3.141592653589793 / 180.0);
    goodcos2 = cg * cg;
  }
  c->goodcos2 = goodcos2;
  std::vector<int> below;  // triangles with an angle below theta (exact)
  const gqm_pt *P = reinterpret_cast<const gqm_pt *>(pts);
  std::unordered_set<uint64_t> segset;
  segset.reserve(2 * (size_t)ns + 8);
  for (int s = 0; s < ns; ++s) segset.insert(ekey(segs[2 * s], segs[2 * s + 1]));
  double minang = 180.0;
  for (int t = 0; t < nt; ++t) {
    int a = tri[3 * t], b = tri[3 * t + 1], d = tri[3 * t + 2];
    if (a < 0 || b < 0 || d < 0 || a >= np || b >= np || d >= np) {
      c->not_ccw++;
      continue;
    }
    if (gqm_orient_exact(P[a].x, P[a].y, P[b].x, P[b].y, P[d].x, P[d].y) <= 0) c->not_ccw++;
    // angles
    int v[3] = {a, b, d};
    double tmin = 180.0;
    for (int i = 0; i < 3; ++i) {
      const gqm_pt &o = P[v[i]], &p = P[v[(i + 1) % 3]], &q = P[v[(i + 2) % 3]];
      double ux = p.x - o.x, uy = p.y - o.y, wx = q.x - o.x, wy = q.y - o.y;
      double ang = atan2(fabs(ux * wy - uy * wx), ux * wx + uy * wy) * (180.0 / 3.141592653589793);
      tmin = std::min(tmin, ang);
    }
    minang = std::min(minang, tmin);
    for (int i = 0; i < 3; ++i)
      if (angle_below(P[v[i]], P[v[(i + 1) % 3]], P[v[(i + 2) % 3]], goodcos2) > 0) {
        c->triangles_below_theta++;
        below.push_back(t);
        break;
      }
    for (int i = 0; i < 3; ++i) {
      int u = v[(i + 1) % 3], w = v[(i + 2) % 3];
      int n = nbr[3 * t + i];
      bool isseg = segset.count(ekey(u, w)) > 0;
      if (n < 0) {
        if (!isseg) c->open_boundary++;
        continue;
      }
      if (n >= nt) {
        c->bad_neighbors++;
        continue;
      }
      // symmetric and sharing the edge
      int j = -1;
      for (int k = 0; k < 3; ++k)
        if (nbr[3 * n + k] == t) j = k;
      if (j < 0) {
        c->bad_neighbors++;
        continue;
      }
      int nu = tri[3 * n + (j + 1) % 3], nw = tri[3 * n + (j + 2) % 3];
      if (!(nu == w && nw == u)) {
        c->bad_neighbors++;
        continue;
      }
      if (isseg || n < t) continue;
      int opp = tri[3 * n + j];
      double r = gqm_incircle_exact(P[a].x, P[a].y, P[b].x, P[b].y, P[d].x, P[d].y, P[opp].x, P[opp].y);
      if (r > 0) c->non_delaunay++;
    }
  }
  c->min_angle_deg = nt ? minang : 0.0;
  // Euler: V - E + F = 2 - L for a connected triangulated domain with L
  // boundary loops (1 for a disk, 1 + h with h holes; F excludes the outer face)
  {
    long long E = 0, B = 0;
    std::vector<int> parent(np > 0 ? np : 1);
    for (int i = 0; i < np; ++i) parent[i] = i;
    auto find = [&](int x) {
      while (parent[x] != x) x = parent[x] = parent[parent[x]];
      return x;
    };
    std::vector<char> onb(np > 0 ? np : 1, 0);
    for (int t = 0; t < nt; ++t)
      for (int i = 0; i < 3; ++i) {
        if (nbr[3 * t + i] < 0) {
          B++;
          const int u = tri[3 * t + (i + 1) % 3], w = tri[3 * t + (i + 2) % 3];
          if (u >= 0 && u < np && w >= 0 && w < np) {
            onb[u] = onb[w] = 1;
            parent[find(u)] = find(w);
          }
        } else {
          E++;
        }
      }
    E = E / 2 + B;
    std::vector<char> used(np, 0);
    for (int t = 0; t < 3 * nt; ++t)
      if (tri[t] >= 0 && tri[t] < np) used[tri[t]] = 1;
    long long V = 0, L = 0;
    for (char u : used) V += u;
    for (int i = 0; i < np; ++i)
      if (onb[i] && find(i) == i) L++;
    if (L == 0) L = 1;
    c->euler_defect = V - E + nt - (2 - L);
  }
  // input points preserved
  for (int i = 0; i < nin && i < np; ++i)
    if (pts[2 * i] != in_pts[2 * i] || pts[2 * i + 1] != in_pts[2 * i + 1]) c->input_points_moved++;
  if (nin > np) c->input_points_moved += nin - np;
  // segment coverage
  std::unordered_map<int, std::vector<int>> adj;
  adj.reserve(2 * (size_t)ns + 8);
  for (int s = 0; s < ns; ++s) {
    adj[segs[2 * s]].push_back(segs[2 * s + 1]);
    adj[segs[2 * s + 1]].push_back(segs[2 * s]);
  }
  double maxdev = 0.0;
  std::unordered_map<int, int> split_of;  // split point -> the input segment it lies on
  for (int s = 0; s < nin_seg; ++s) {
    int a = in_segs[2 * s], b = in_segs[2 * s + 1];
    double lx = P[b].x - P[a].x, ly = P[b].y - P[a].y, len2 = lx * lx + ly * ly;
    int cur = a, prev = -1;
    bool ok = false;
    for (int guard = 0; guard < 1 << 22; ++guard) {
      if (cur == b) {
        ok = true;
        break;
      }
      if (cur != a) split_of[cur] = s;
      auto it = adj.find(cur);
      if (it == adj.end()) break;
      int nxt = -1;
      double best = 0.0;
      for (int w : it->second) {
        if (w == prev) continue;
        double fwd = (P[w].x - P[cur].x) * lx + (P[w].y - P[cur].y) * ly;
        if (fwd <= 0) continue;
        double dev = fabs((P[w].x - P[a].x) * ly - (P[w].y - P[a].y) * lx) / len2;
        if (nxt < 0 || dev < best) {
          nxt = w;
          best = dev;
        }
      }
      if (nxt < 0 || best > 1e-6) break;
      maxdev = std::max(maxdev, best);
      prev = cur;
      cur = nxt;
    }
    if (!ok) c->segments_missing++;
  }
  c->max_segment_deviation = maxdev;
  // the reference's exemption for every triangle below theta
  for (int t : below) {
    const int v[3] = {tri[3 * t], tri[3 * t + 1], tri[3 * t + 2]};
    // shortest edge: edge i joins v[i+1] and v[i+2]; ties go as in
    // kernelComputeSmallestAngle (refine.cu:317-374): edge 0, then 1, else 2
    const Exp l0 = ex_dist2(P[v[1]], P[v[2]]), l1 = ex_dist2(P[v[2]], P[v[0]]), l2 = ex_dist2(P[v[0]], P[v[1]]);
    auto less = [](const Exp &x, const Exp &y) { return ex_sign(ex_add(x, ex_neg(y))) < 0; };
    int sh = 2;
    if (less(l0, l1) && less(l0, l2))
      sh = 0;
    else if (less(l1, l0) && less(l1, l2))
      sh = 1;
    const int vo = v[(sh + 1) % 3], vd = v[(sh + 2) % 3];
    bool exempt = false;
    auto io = split_of.find(vo), id = split_of.find(vd);
    if (!segset.count(ekey(vo, vd)) && io != split_of.end() && id != split_of.end()) {
      const int g1x = in_segs[2 * io->second], g1y = in_segs[2 * io->second + 1];
      const int g2x = in_segs[2 * id->second], g2y = in_segs[2 * id->second + 1];
      int common = -1;
      if (g1x == g2x || g1x == g2y)
        common = g1x;
      else if (g1y == g2x || g1y == g2y)
        common = g1y;
      if (common >= 0) {
        const Exp d1 = ex_dist2(P[common], P[vo]), d2 = ex_dist2(P[common], P[vd]);
        exempt = ex_sign(ex_add(ex_scale(d2, 1.001), ex_neg(d1))) > 0 &&
                 ex_sign(ex_add(d1, ex_neg(ex_scale(d2, 0.999)))) > 0;
      }
    }
    if (exempt)
      c->exempted++;
    else if (reference_tie_passes(P[v[0]], P[v[1]], P[v[2]], goodcos2))
      c->tie_passed++;
    else
      c->quality_violations++;
  }
  return (c->not_ccw || c->bad_neighbors || c->open_boundary || c->non_delaunay || c->segments_missing ||
          c->input_points_moved || c->euler_defect || c->quality_violations)
             ? 1
             : 0;
}

}  // extern "C"

// Predicate entry points for the predicate tests (points as x, y pairs).
extern "C" {
double gqm_pred_orient_exact(const double *a, const double *b, const double *c) {
  return gqm_orient_exact(a[0], a[1], b[0], b[1], c[0], c[1]);
}
double gqm_pred_incircle_exact(const double *a, const double *b, const double *c, const double *d) {
  return gqm_incircle_exact(a[0], a[1], b[0], b[1], c[0], c[1], d[0], d[1]);
}
double gqm_pred_orient_ref(const double *a, const double *b, const double *c) {
  return gqm_orient_ref(a[0], a[1], b[0], b[1], c[0], c[1]);
}
double gqm_pred_incircle_ref_fallback(const double *a, const double *b, const double *c, const double *d) {
  return gqm_incircle_zero_fallback_ref(a[0], a[1], b[0], b[1], c[0], c[1], d[0], d[1]);
}
}
