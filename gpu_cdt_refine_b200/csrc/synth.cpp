// Seeded synthetic PSLG generators for the benchmark workloads.
//
// The reference generates its inputs with GenerateRandomInput
// (GPU_Refine/mesh.cpp:49-400): random points, then random point pairs kept as
// segments when they pass a rejection test, then Triangle's CDT.  The
// workloads used here have their own distributions (uniform square, mixture
// of isotropic Gaussians, jittered grid plus concentric circles), but keep the
// reference's rejection idea with exact predicates:
//   * a candidate segment joins two distinct input points;
//   * neither endpoint is an endpoint of an earlier segment or a convex hull
//     vertex (hull edges become segments in the CDT, so a shared endpoint
//     would create an uncontrolled small input angle);
//   * it crosses no earlier segment (exact orient2d);
//   * no other input point lies on it (exact orient2d);
//   * like the reference's length cap (mesh.cpp:247-248), pairs are drawn
//     between nearby points: the second endpoint is a near neighbour of the
//     first in Hilbert-curve order, so the rejection loop terminates.
// Random numbers come from SplitMix64, so outputs are identical on every
// machine for a given seed.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <unordered_map>
#include <vector>

#include "predicates.h"

namespace {

struct Rng {
  uint64_t s;
  explicit Rng(uint64_t seed) : s(seed) {}
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double uni() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }  // [0,1)
  double gauss() {                                                                // Box-Muller
    double u1 = uni(), u2 = uni();
    if (u1 < 1e-300) u1 = 1e-300;
    return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
  }
  uint64_t below(uint64_t n) { return next() % n; }
};

uint64_t hilbert_d(uint32_t x, uint32_t y) {
  const uint32_t n = 1u << 16;
  uint64_t d = 0;
  for (uint32_t s = n / 2; s > 0; s /= 2) {
    uint32_t rx = (x & s) > 0, ry = (y & s) > 0;
    d += (uint64_t)s * s * ((3 * rx) ^ ry);
    if (ry == 0) {
      if (rx == 1) {
        x = s - 1 - x;
        y = s - 1 - y;
      }
      std::swap(x, y);
    }
  }
  return d;
}

inline double orient(const gqm_pt *P, int a, int b, int c) {
  return gqm_orient_exact(P[a].x, P[a].y, P[b].x, P[b].y, P[c].x, P[c].y);
}

std::vector<char> hull_marks(const gqm_pt *P, int np) {
  std::vector<int> idx(np);
  for (int i = 0; i < np; ++i) idx[i] = i;
  std::sort(idx.begin(), idx.end(),
            [&](int a, int b) { return P[a].x < P[b].x || (P[a].x == P[b].x && P[a].y < P[b].y); });
  std::vector<int> H(2 * np + 2);
  int k = 0;
  for (int i = 0; i < np; ++i) {
    while (k >= 2 && orient(P, H[k - 2], H[k - 1], idx[i]) <= 0) --k;
    H[k++] = idx[i];
  }
  for (int i = np - 2, t = k + 1; i >= 0; --i) {
    while (k >= t && orient(P, H[k - 2], H[k - 1], idx[i]) <= 0) --k;
    H[k++] = idx[i];
  }
  std::vector<char> m(np, 0);
  for (int i = 0; i < k; ++i) m[H[i]] = 1;
  return m;
}

// Uniform hash grid over points and accepted segments.
struct Grid {
  double x0, y0, h;
  std::unordered_map<uint64_t, std::vector<int>> pts, segs;
  uint64_t key(long cx, long cy) const { return ((uint64_t)(uint32_t)cx << 32) | (uint32_t)cy; }
  long cx(double x) const { return (long)floor((x - x0) / h); }
  long cy(double y) const { return (long)floor((y - y0) / h); }
  // conservative set of cells touched by segment p-q
  void cells(const gqm_pt &p, const gqm_pt &q, std::vector<uint64_t> &out) const {
    out.clear();
    double len = sqrt((q.x - p.x) * (q.x - p.x) + (q.y - p.y) * (q.y - p.y));
    int steps = (int)ceil(len / (0.25 * h)) + 1;
    long lx = LONG_MIN, ly = LONG_MIN;
    for (int s = 0; s <= steps; ++s) {
      double t = (double)s / steps;
      long a = cx(p.x + t * (q.x - p.x)), b = cy(p.y + t * (q.y - p.y));
      if (a == lx && b == ly) continue;
      lx = a;
      ly = b;
      for (int dx = -1; dx <= 1; ++dx)
        for (int dy = -1; dy <= 1; ++dy) out.push_back(key(a + dx, b + dy));
    }
    std::sort(out.begin(), out.end());
    out.erase(std::unique(out.begin(), out.end()), out.end());
  }
};

struct Picker {
  const gqm_pt *P;
  int np;
  Grid g;
  std::vector<char> used;  // endpoint of a kept segment, or hull vertex
  std::vector<int> kept;
  std::vector<uint64_t> tmp;

  void init(const gqm_pt *P_, int np_, int exclude_hull) {
    P = P_;
    np = np_;
    double x0 = P[0].x, x1 = P[0].x, y0 = P[0].y, y1 = P[0].y;
    for (int i = 1; i < np; ++i) {
      x0 = std::min(x0, P[i].x);
      x1 = std::max(x1, P[i].x);
      y0 = std::min(y0, P[i].y);
      y1 = std::max(y1, P[i].y);
    }
    double area = std::max((x1 - x0) * (y1 - y0), 1e-300);
    g.x0 = x0;
    g.y0 = y0;
    g.h = 0.25 * sqrt(area / np);
    if (!(g.h > 0)) g.h = 1.0;
    for (int i = 0; i < np; ++i) g.pts[g.key(g.cx(P[i].x), g.cy(P[i].y))].push_back(i);
    used.assign(np, 0);
    if (exclude_hull) used = hull_marks(P, np);
  }

  static bool cross(const gqm_pt *P, int p, int q, int r, int s) {
    double o1 = orient(P, p, q, r), o2 = orient(P, p, q, s);
    if ((o1 > 0 && o2 > 0) || (o1 < 0 && o2 < 0)) return false;
    double o3 = orient(P, r, s, p), o4 = orient(P, r, s, q);
    if ((o3 > 0 && o4 > 0) || (o3 < 0 && o4 < 0)) return false;
    return true;  // proper crossing, touching or collinear overlap
  }

  bool try_add(int p, int q) {
    if (p == q || used[p] || used[q]) return false;
    g.cells(P[p], P[q], tmp);
    double bx0 = std::min(P[p].x, P[q].x), bx1 = std::max(P[p].x, P[q].x);
    double by0 = std::min(P[p].y, P[q].y), by1 = std::max(P[p].y, P[q].y);
    for (uint64_t k : tmp) {
      auto it = g.segs.find(k);
      if (it != g.segs.end())
        for (int s : it->second)
          if (cross(P, p, q, kept[2 * s], kept[2 * s + 1])) return false;
      auto jt = g.pts.find(k);
      if (jt != g.pts.end())
        for (int r : jt->second) {
          if (r == p || r == q) continue;
          if (P[r].x < bx0 || P[r].x > bx1 || P[r].y < by0 || P[r].y > by1) continue;
          if (orient(P, p, q, r) == 0) return false;
        }
    }
    int sid = (int)kept.size() / 2;
    kept.push_back(p);
    kept.push_back(q);
    used[p] = used[q] = 1;
    for (uint64_t k : tmp) g.segs[k].push_back(sid);
    return true;
  }
};

std::vector<int> hilbert_order(const gqm_pt *P, int np) {
  double x0 = P[0].x, x1 = P[0].x, y0 = P[0].y, y1 = P[0].y;
  for (int i = 1; i < np; ++i) {
    x0 = std::min(x0, P[i].x);
    x1 = std::max(x1, P[i].x);
    y0 = std::min(y0, P[i].y);
    y1 = std::max(y1, P[i].y);
  }
  double sx = (x1 > x0) ? 65535.0 / (x1 - x0) : 0.0, sy = (y1 > y0) ? 65535.0 / (y1 - y0) : 0.0;
  std::vector<std::pair<uint64_t, int>> key(np);
  for (int i = 0; i < np; ++i)
    key[i] = {hilbert_d((uint32_t)((P[i].x - x0) * sx), (uint32_t)((P[i].y - y0) * sy)), i};
  std::sort(key.begin(), key.end());
  std::vector<int> ord(np);
  for (int i = 0; i < np; ++i) ord[i] = key[i].second;
  return ord;
}

int dedup(double *xy, int n) {  // exact duplicates removed, first occurrence kept
  std::vector<int> idx(n);
  for (int i = 0; i < n; ++i) idx[i] = i;
  std::sort(idx.begin(), idx.end(), [&](int a, int b) {
    if (xy[2 * a] != xy[2 * b]) return xy[2 * a] < xy[2 * b];
    if (xy[2 * a + 1] != xy[2 * b + 1]) return xy[2 * a + 1] < xy[2 * b + 1];
    return a < b;
  });
  std::vector<char> drop(n, 0);
  for (int i = 1; i < n; ++i)
    if (xy[2 * idx[i]] == xy[2 * idx[i - 1]] && xy[2 * idx[i] + 1] == xy[2 * idx[i - 1] + 1]) drop[idx[i]] = 1;
  int m = 0;
  for (int i = 0; i < n; ++i)
    if (!drop[i]) {
      xy[2 * m] = xy[2 * i];
      xy[2 * m + 1] = xy[2 * i + 1];
      ++m;
    }
  return m;
}

}  // namespace

extern "C" {

// Points uniform in [lo, hi]^2.  Returns the count after removing duplicates.
int gqm_synth_uniform(int n, double lo, double hi, uint64_t seed, double *xy) {
  Rng r(seed);
  for (int i = 0; i < n; ++i) {
    xy[2 * i] = lo + (hi - lo) * r.uni();
    xy[2 * i + 1] = lo + (hi - lo) * r.uni();
  }
  return dedup(xy, n);
}

// Mixture of k isotropic Gaussians (centres uniform in [0,L]^2, sigma
// log-uniform in [smin, smax], equal weights) plus a fraction `bg` of uniform
// background points in [0,L]^2.  Points outside [0,L]^2 are redrawn.
int gqm_synth_clusters(int n, int k, double L, double smin, double smax, double bg, uint64_t seed, double *xy) {
  Rng r(seed);
  std::vector<double> cx(k), cy(k), sg(k);
  for (int j = 0; j < k; ++j) {
    cx[j] = L * r.uni();
    cy[j] = L * r.uni();
    sg[j] = exp(log(smin) + (log(smax) - log(smin)) * r.uni());
  }
  int nbg = (int)llround(bg * n);
  for (int i = 0; i < n; ++i) {
    double x, y;
    if (i < nbg) {
      x = L * r.uni();
      y = L * r.uni();
    } else {
      int j = (int)r.below((uint64_t)k);
      do {
        x = cx[j] + sg[j] * r.gauss();
        y = cy[j] + sg[j] * r.gauss();
      } while (x < 0 || x > L || y < 0 || y > L);
    }
    xy[2 * i] = x;
    xy[2 * i + 1] = y;
  }
  return dedup(xy, n);
}

// Adversarial structure: a g x g grid (spacing sp) with each coordinate
// jittered uniformly by +-jit*sp, followed by `nc` concentric circles about
// (cxy, cxy) with radii evenly spaced in [r0, r1] and `per` points each
// (equal angular spacing, random phase per circle).  circle_id receives the
// circle index of each point (-1 for grid points).  Returns the count.
int gqm_synth_grid_circles(int g, double sp, double jit, int nc, int per, double cxy, double r0, double r1,
                           uint64_t seed, double *xy, int *circle_id) {
  Rng r(seed);
  int m = 0;
  for (int i = 0; i < g; ++i)
    for (int j = 0; j < g; ++j) {
      xy[2 * m] = i * sp + (2.0 * r.uni() - 1.0) * jit * sp;
      xy[2 * m + 1] = j * sp + (2.0 * r.uni() - 1.0) * jit * sp;
      circle_id[m] = -1;
      ++m;
    }
  for (int c = 0; c < nc; ++c) {
    double rad = (nc > 1) ? r0 + (r1 - r0) * c / (nc - 1) : r0;
    double ph = 6.283185307179586 * r.uni();
    for (int k = 0; k < per; ++k) {
      double a = ph + 6.283185307179586 * k / per;
      xy[2 * m] = cxy + rad * cos(a);
      xy[2 * m + 1] = cxy + rad * sin(a);
      circle_id[m] = c;
      ++m;
    }
  }
  // keep circle ids aligned with the deduplicated order
  std::vector<double> tmp(xy, xy + 2 * (size_t)m);
  std::vector<int> cid(circle_id, circle_id + m);
  int n2 = dedup(xy, m);
  if (n2 != m) {  // recompute ids by matching (rare: exact duplicates)
    std::unordered_map<uint64_t, int> pos;
    for (int i = 0; i < m; ++i) {
      uint64_t hx, hy;
      memcpy(&hx, &tmp[2 * i], 8);
      memcpy(&hy, &tmp[2 * i + 1], 8);
      pos[hx * 1000003ull ^ hy] = cid[i];
    }
    for (int i = 0; i < n2; ++i) {
      uint64_t hx, hy;
      memcpy(&hx, &xy[2 * i], 8);
      memcpy(&hy, &xy[2 * i + 1], 8);
      circle_id[i] = pos[hx * 1000003ull ^ hy];
    }
  }
  return n2;
}

// Random nearby-pair segments (rules in the file header).  Pairs are
// (ord[i], ord[i+gap]) in Hilbert order with i uniform and gap uniform in
// [1, max_gap].  Stops after nseg segments or max_tries candidates.
// Returns the number of segments written to segs (2 ints each).
int gqm_pick_segments(int np, const double *pts, int nseg, int max_gap, uint64_t seed, long long max_tries,
                      int *segs) {
  const gqm_pt *P = reinterpret_cast<const gqm_pt *>(pts);
  Picker pk;
  pk.init(P, np, 1);
  std::vector<int> ord = hilbert_order(P, np);
  Rng r(seed);
  for (long long t = 0; t < max_tries && (int)pk.kept.size() / 2 < nseg; ++t) {
    int i = (int)r.below((uint64_t)np);
    int gap = 1 + (int)r.below((uint64_t)max_gap);
    if (i + gap >= np) continue;
    pk.try_add(ord[i], ord[i + gap]);
  }
  memcpy(segs, pk.kept.data(), sizeof(int) * pk.kept.size());
  return (int)pk.kept.size() / 2;
}

// Keep, in order, the candidate segments that pass the same rules.
int gqm_filter_segments(int np, const double *pts, int ncand, const int *cand, int nseg, int *segs) {
  const gqm_pt *P = reinterpret_cast<const gqm_pt *>(pts);
  Picker pk;
  pk.init(P, np, 1);
  for (int c = 0; c < ncand && (int)pk.kept.size() / 2 < nseg; ++c) pk.try_add(cand[2 * c], cand[2 * c + 1]);
  memcpy(segs, pk.kept.data(), sizeof(int) * pk.kept.size());
  return (int)pk.kept.size() / 2;
}

}  // extern "C"
