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
//   5. minimum angle statistics (degrees, FP64 atan2 of exact-enough
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
};

static inline uint64_t ekey(int a, int b) {
  uint32_t lo = (uint32_t)std::min(a, b), hi = (uint32_t)std::max(a, b);
  return ((uint64_t)hi << 32) | lo;
}

int gqm_certify(int np, const double *pts, int nt, const int *tri, const int *nbr, int ns, const int *segs,
                int nin, const double *in_pts, int nin_seg, const int *in_segs, double theta,
                gqm_certificate *c) {
  memset(c, 0, sizeof(*c));
  c->theta = theta;
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
    if (tmin < theta * (1.0 - 1e-9)) c->triangles_below_theta++;
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
  return (c->not_ccw || c->bad_neighbors || c->open_boundary || c->non_delaunay || c->segments_missing ||
          c->input_points_moved || c->euler_defect)
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
