// Input construction for the refiner: constrained Delaunay triangulation of a
// planar straight-line graph, and the synthetic segment pickers used by the
// benchmark inputs.
//
// The refiner's input contract (GPU_Refine/refine.h:385-386, README
// "triangulateio *input") is a CDT in Triangle's triangulateio layout with
// zero-based indices, counterclockwise triangles, neighbour j opposite vertex
// j (-1 on the boundary), and the convex hull enclosed by segments (Triangle's
// "pzQnc" switches, GPU_Refine/mesh.cpp:397).  gqm_cdt_build produces exactly
// that, without Triangle:
//   * Delaunay triangulation by incremental Bowyer-Watson insertion in
//     Hilbert-curve order with ghost triangles for the exterior, so the convex
//     hull comes out exact;
//   * each segment missing from the triangulation is inserted by removing the
//     triangles it crosses and re-triangulating the two pseudo-polygons on
//     either side with the recursive Delaunay-vertex rule;
//   * every hull edge that is not already a segment becomes a segment.
// All decisions use the exact predicates of predicates.h.
//
// Preconditions (checked, error code on violation): no duplicate points, no
// segment passes through a point, no two segments cross.
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <unordered_map>
#include <vector>

#include "gqm_cdt.h"
#include "predicates.h"

namespace {

struct Tri {
  int v[3];  // -1 marks the ghost vertex at infinity
  int n[3];  // neighbour across the edge opposite v[i]
};

inline double orient(const gqm_pt *P, int a, int b, int c) {
  return gqm_orient_exact(P[a].x, P[a].y, P[b].x, P[b].y, P[c].x, P[c].y);
}
inline double incircle(const gqm_pt *P, int a, int b, int c, int d) {
  return gqm_incircle_exact(P[a].x, P[a].y, P[b].x, P[b].y, P[c].x, P[c].y, P[d].x, P[d].y);
}

// Hilbert index of (x, y) in a 2^16 x 2^16 grid.
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
  for (int i = 0; i < np; ++i) {
    uint32_t hx = (uint32_t)((P[i].x - x0) * sx), hy = (uint32_t)((P[i].y - y0) * sy);
    key[i] = {hilbert_d(hx, hy), i};
  }
  std::sort(key.begin(), key.end());
  std::vector<int> ord(np);
  for (int i = 0; i < np; ++i) ord[i] = key[i].second;
  return ord;
}

struct Builder {
  const gqm_pt *P;
  int np;
  std::vector<Tri> T;
  std::vector<char> dead;
  std::vector<int> freelist;
  std::vector<int> vtri;  // some live triangle incident to each vertex
  int last = 0;           // walk start
  uint32_t rng = 12345;

  int alloc() {
    if (!freelist.empty()) {
      int t = freelist.back();
      freelist.pop_back();
      dead[t] = 0;
      return t;
    }
    T.push_back(Tri());
    dead.push_back(0);
    return (int)T.size() - 1;
  }
  void kill(int t) {
    dead[t] = 1;
    freelist.push_back(t);
  }
  static bool ghost(const Tri &t) { return t.v[0] < 0 || t.v[1] < 0 || t.v[2] < 0; }
  void touch(int t) {
    for (int i = 0; i < 3; ++i)
      if (T[t].v[i] >= 0) vtri[T[t].v[i]] = t;
  }
  int edge_index(int t, int a, int b) const {  // index i such that edge opposite v[i] is {a,b}
    for (int i = 0; i < 3; ++i) {
      int u = T[t].v[(i + 1) % 3], w = T[t].v[(i + 2) % 3];
      if ((u == a && w == b) || (u == b && w == a)) return i;
    }
    return -1;
  }

  // Conflict test for Bowyer-Watson.
  bool conflict(int t, int p) const {
    const Tri &r = T[t];
    for (int k = 0; k < 3; ++k) {
      if (r.v[k] < 0) {
        int u = r.v[(k + 1) % 3], w = r.v[(k + 2) % 3];
        double o = orient(P, u, w, p);
        if (o > 0) return true;
        if (o < 0) return false;
        // collinear with the hull edge: conflict iff strictly between u and w
        double dx = P[w].x - P[u].x, dy = P[w].y - P[u].y;
        double t0 = (P[p].x - P[u].x) * dx + (P[p].y - P[u].y) * dy;
        double t1 = (P[p].x - P[w].x) * dx + (P[p].y - P[w].y) * dy;
        return t0 > 0 && t1 < 0;
      }
    }
    return incircle(P, r.v[0], r.v[1], r.v[2], p) > 0;
  }

  // Visibility walk to a triangle containing p (or a ghost whose hull edge
  // sees p).  Returns -1 if the walk does not finish (degenerate input).
  int locate(int p) {
    int t = last;
    if (t < 0 || t >= (int)T.size() || dead[t] || ghost(T[t])) {
      t = -1;
      for (int i = 0; i < (int)T.size(); ++i)
        if (!dead[i] && !ghost(T[i])) {
          t = i;
          break;
        }
    }
    for (long it = 0; it < 4L * (long)T.size() + 64; ++it) {
      const Tri &r = T[t];
      if (ghost(r)) return t;
      rng = rng * 1664525u + 1013904223u;
      int s = (rng >> 16) % 3;
      bool moved = false;
      for (int q = 0; q < 3; ++q) {
        int i = (s + q) % 3;
        int u = r.v[(i + 1) % 3], w = r.v[(i + 2) % 3];
        if (orient(P, u, w, p) < 0) {
          t = r.n[i];
          moved = true;
          break;
        }
      }
      if (!moved) return t;
    }
    return -1;
  }

  int insert_point(int p) {
    int t0 = locate(p);
    if (t0 < 0) return -1;
    // grow cavity
    std::vector<int> cav, stack{t0};
    std::vector<int> mark;  // reuse dead[] as scratch is unsafe; keep small vectors
    auto in_cav = [&](int t) { return std::find(cav.begin(), cav.end(), t) != cav.end(); };
    cav.push_back(t0);
    while (!stack.empty()) {
      int t = stack.back();
      stack.pop_back();
      for (int i = 0; i < 3; ++i) {
        int nb = T[t].n[i];
        if (nb < 0 || in_cav(nb)) continue;
        if (conflict(nb, p)) {
          cav.push_back(nb);
          stack.push_back(nb);
        }
      }
    }
    // boundary edges
    struct BE {
      int a, b, out, outi;
    };
    std::vector<BE> be;
    for (int t : cav)
      for (int i = 0; i < 3; ++i) {
        int nb = T[t].n[i];
        if (nb >= 0 && in_cav(nb)) continue;
        BE e{T[t].v[(i + 1) % 3], T[t].v[(i + 2) % 3], nb, -1};
        if (nb >= 0) e.outi = edge_index(nb, e.a, e.b);
        be.push_back(e);
      }
    for (int t : cav) kill(t);
    std::vector<int> nt(be.size());
    for (size_t k = 0; k < be.size(); ++k) {
      int t = alloc();
      nt[k] = t;
      T[t].v[0] = be[k].a;
      T[t].v[1] = be[k].b;
      T[t].v[2] = p;
      T[t].n[2] = be[k].out;
      if (be[k].out >= 0) T[be[k].out].n[be[k].outi] = t;
    }
    // link the fan: triangle (a,b,p) meets (b,c,p) across (b,p), i.e. its n[0];
    // and (z,a,p) across (p,a), i.e. its n[1].
    for (size_t k = 0; k < be.size(); ++k) {
      for (size_t m = 0; m < be.size(); ++m) {
        if (be[m].a == be[k].b) {
          T[nt[k]].n[0] = nt[m];
          T[nt[m]].n[1] = nt[k];
        }
      }
    }
    for (int t : nt) touch(t);
    for (int t : nt)
      if (!ghost(T[t])) {
        last = t;
        break;
      }
    return 0;
  }

  int build_dt(const std::vector<int> &ord) {
    vtri.assign(np, -1);
    // initial triangle: first point, then first two making a non-degenerate triangle
    int a = ord[0], b = -1, c = -1, ib = -1, ic = -1;
    for (int i = 1; i < np; ++i)
      if (P[ord[i]].x != P[a].x || P[ord[i]].y != P[a].y) {
        b = ord[i];
        ib = i;
        break;
      }
    if (b < 0) return -2;
    for (int i = 1; i < np; ++i) {
      if (i == ib) continue;
      if (orient(P, a, b, ord[i]) != 0) {
        c = ord[i];
        ic = i;
        break;
      }
    }
    if (c < 0) return -2;  // all collinear
    if (orient(P, a, b, c) < 0) std::swap(b, c);
    int t = alloc(), g0 = alloc(), g1 = alloc(), g2 = alloc();
    T[t] = Tri{{a, b, c}, {g1, g2, g0}};
    // ghost across edge opposite v[i] of t: edge (v[i+1], v[i+2]) reversed
    T[g0] = Tri{{b, a, -1}, {-1, -1, t}};  // across (a,b)
    T[g1] = Tri{{c, b, -1}, {-1, -1, t}};  // across (b,c)
    T[g2] = Tri{{a, c, -1}, {-1, -1, t}};  // across (c,a)
    // ghost-ghost links: (b,a,inf).n[0] is across (a,inf) -> ghost (a,c,inf)
    T[g0].n[0] = g2;
    T[g2].n[1] = g0;
    T[g0].n[1] = g1;
    T[g1].n[0] = g0;
    T[g1].n[1] = g2;
    T[g2].n[0] = g1;
    touch(t);
    touch(g0);
    touch(g1);
    touch(g2);
    last = t;
    for (int i = 1; i < np; ++i) {
      if (i == ib || i == ic) continue;
      if (insert_point(ord[i]) != 0) return -3;
    }
    return 0;
  }

  // Find the edge {a,b}; returns triangle and edge index or -1.
  int find_edge(int a, int b, int *ei) {
    int t0 = vtri[a];
    int t = t0;
    for (int guard = 0; guard < 100000; ++guard) {
      int i = -1;
      for (int k = 0; k < 3; ++k)
        if (T[t].v[k] == a) i = k;
      if (i < 0) return -1;
      for (int k = 0; k < 3; ++k)
        if (T[t].v[k] == b) {
          *ei = 3 - i - k;
          return t;
        }
      t = T[t].n[(i + 1) % 3];  // rotate around a
      if (t == t0 || t < 0) return -1;
    }
    return -1;
  }

  // Recursive Delaunay re-triangulation of the pseudo-polygon a, chain..., b
  // lying to the left of a->b.  Created triangles are appended to out.
  void fill(int a, int b, const int *ch, int m, std::vector<int> &out) {
    if (m == 0) return;
    int k = 0;
    for (int j = 1; j < m; ++j)
      if (incircle(P, a, b, ch[k], ch[j]) > 0) k = j;
    int t = alloc();
    T[t].v[0] = a;
    T[t].v[1] = b;
    T[t].v[2] = ch[k];
    T[t].n[0] = T[t].n[1] = T[t].n[2] = -1;
    out.push_back(t);
    fill(a, ch[k], ch, k, out);
    fill(ch[k], b, ch + k + 1, m - k - 1, out);
  }

  int insert_segment(int a, int b) {
    int ei;
    if (a == b) return -4;
    if (find_edge(a, b, &ei) >= 0) return 0;
    // triangle in a's fan whose angle contains the direction of b
    int t0 = vtri[a], t = t0, start = -1, ia = -1;
    for (int guard = 0; guard < 100000; ++guard) {
      int i = -1;
      for (int k = 0; k < 3; ++k)
        if (T[t].v[k] == a) i = k;
      if (i < 0) return -5;
      if (!ghost(T[t])) {
        int u = T[t].v[(i + 1) % 3], w = T[t].v[(i + 2) % 3];
        if (orient(P, a, u, b) > 0 && orient(P, a, w, b) < 0) {
          start = t;
          ia = i;
          break;
        }
      }
      t = T[t].n[(i + 1) % 3];
      if (t == t0 || t < 0) break;
    }
    if (start < 0) return -5;
    std::vector<int> crossed{start}, left, right;
    int u = T[start].v[(ia + 1) % 3], w = T[start].v[(ia + 2) % 3];  // u right of a->b? check below
    // orient(a,u,b) > 0 means b is left of a->u, i.e. u is right of a->b.
    int R = u, L = w;
    int cur = start, ce = ia;  // crossing edge is opposite v[ce] of cur: (R, L)
    right.push_back(R);
    left.push_back(L);
    for (int guard = 0; guard < 1000000; ++guard) {
      int nb = T[cur].n[ce];
      if (nb < 0 || ghost(T[nb])) return -6;
      int j = edge_index(nb, R, L);
      int x = T[nb].v[j];
      crossed.push_back(nb);
      if (x == b) break;
      double o = orient(P, a, b, x);
      if (o == 0) return -7;  // a point on the segment
      if (o > 0) {
        L = x;
        left.push_back(x);
      } else {
        R = x;
        right.push_back(x);
      }
      cur = nb;
      ce = edge_index(cur, R, L);
      if (ce < 0) return -6;
    }
    // boundary edges of the union of crossed triangles, with their outside neighbours
    struct OE {
      int a, b, out, outi;
    };
    std::vector<OE> outer;
    auto is_crossed = [&](int q) { return std::find(crossed.begin(), crossed.end(), q) != crossed.end(); };
    for (int q : crossed)
      for (int i = 0; i < 3; ++i) {
        int nb = T[q].n[i];
        if (nb >= 0 && is_crossed(nb)) continue;
        OE e{T[q].v[(i + 1) % 3], T[q].v[(i + 2) % 3], nb, -1};
        if (nb >= 0) e.outi = edge_index(nb, e.a, e.b);
        outer.push_back(e);
      }
    for (int q : crossed) kill(q);
    std::vector<int> made;
    // left polygon: a, left..., b lies to the left of a->b -> triangles (a,b,c)
    fill(a, b, left.data(), (int)left.size(), made);
    // right polygon lies to the left of b->a; chain in order from b to a
    std::vector<int> rr(right.rbegin(), right.rend());
    fill(b, a, rr.data(), (int)rr.size(), made);
    // link: key by undirected edge
    std::unordered_map<uint64_t, std::pair<int, int>> open;
    auto key = [](int x, int y) {
      uint32_t lo = (uint32_t)std::min(x, y), hi = (uint32_t)std::max(x, y);
      return ((uint64_t)hi << 32) | lo;
    };
    for (const OE &e : outer) open[key(e.a, e.b)] = {-2 - (int)(&e - &outer[0]), 0};
    for (int q : made)
      for (int i = 0; i < 3; ++i) {
        int x = T[q].v[(i + 1) % 3], y = T[q].v[(i + 2) % 3];
        uint64_t k = key(x, y);
        auto it = open.find(k);
        if (it == open.end()) {
          open[k] = {q, i};
        } else {
          int o = it->second.first;
          if (o <= -2) {
            const OE &e = outer[-2 - o];
            T[q].n[i] = e.out;
            if (e.out >= 0) T[e.out].n[e.outi] = q;
          } else {
            T[q].n[i] = o;
            T[o].n[it->second.second] = q;
          }
          open.erase(it);
        }
      }
    for (int q : made) touch(q);
    return 0;
  }
};

}  // namespace

extern "C" {

// Constrained Delaunay triangulation with the convex hull enclosed by
// segments (the contract of Triangle's "pzQnc", GPU_Refine/mesh.cpp:397).
// Output segments: the input segments first, in input order, then every hull
// edge that is not an input segment.  Returns 0 on success.
int gqm_cdt_build(int np, const double *pts, int ns, const int *segs, gqm_cdt_result *out) {
  memset(out, 0, sizeof(*out));
  if (np < 3) return out->status = -1;
  const gqm_pt *P = reinterpret_cast<const gqm_pt *>(pts);
  {  // duplicates
    std::vector<int> idx(np);
    for (int i = 0; i < np; ++i) idx[i] = i;
    std::sort(idx.begin(), idx.end(),
              [&](int a, int b) { return P[a].x < P[b].x || (P[a].x == P[b].x && P[a].y < P[b].y); });
    for (int i = 1; i < np; ++i)
      if (P[idx[i]].x == P[idx[i - 1]].x && P[idx[i]].y == P[idx[i - 1]].y) return out->status = -8;
  }
  Builder B;
  B.P = P;
  B.np = np;
  B.T.reserve(2 * (size_t)np + 16);
  std::vector<int> ord = hilbert_order(P, np);
  int rc = B.build_dt(ord);
  if (rc) return out->status = rc;
  std::vector<char> isseg;  // unused: constraint set is implicit in output list
  for (int s = 0; s < ns; ++s) {
    rc = B.insert_segment(segs[2 * s], segs[2 * s + 1]);
    if (rc) return out->status = rc;
  }
  // compact: real triangles in storage order
  std::vector<int> newid(B.T.size(), -1);
  int nt = 0;
  for (size_t t = 0; t < B.T.size(); ++t)
    if (!B.dead[t] && !Builder::ghost(B.T[t])) newid[t] = nt++;
  out->numberofpoints = np;
  out->numberoftriangles = nt;
  out->trianglelist = (int *)malloc(sizeof(int) * 3 * (size_t)nt);
  out->neighborlist = (int *)malloc(sizeof(int) * 3 * (size_t)nt);
  for (size_t t = 0; t < B.T.size(); ++t) {
    int id = newid[t];
    if (id < 0) continue;
    for (int i = 0; i < 3; ++i) {
      out->trianglelist[3 * id + i] = B.T[t].v[i];
      int nb = B.T[t].n[i];
      out->neighborlist[3 * id + i] = (nb >= 0) ? newid[nb] : -1;
    }
  }
  // segments: input, then hull edges not already present
  std::unordered_map<uint64_t, int> have;
  auto key = [](int x, int y) {
    uint32_t lo = (uint32_t)std::min(x, y), hi = (uint32_t)std::max(x, y);
    return ((uint64_t)hi << 32) | lo;
  };
  std::vector<int> S;
  S.reserve(2 * (size_t)ns + 64);
  for (int s = 0; s < ns; ++s) {
    uint64_t k = key(segs[2 * s], segs[2 * s + 1]);
    if (have.count(k)) continue;
    have[k] = 1;
    S.push_back(segs[2 * s]);
    S.push_back(segs[2 * s + 1]);
  }
  for (size_t t = 0; t < B.T.size(); ++t) {
    int id = newid[t];
    if (id < 0) continue;
    for (int i = 0; i < 3; ++i)
      if (out->neighborlist[3 * id + i] < 0) {
        int u = B.T[t].v[(i + 1) % 3], w = B.T[t].v[(i + 2) % 3];
        uint64_t k = key(u, w);
        if (have.count(k)) continue;
        have[k] = 1;
        S.push_back(u);
        S.push_back(w);
      }
  }
  out->numberofsegments = (int)(S.size() / 2);
  out->segmentlist = (int *)malloc(sizeof(int) * S.size() + 8);
  memcpy(out->segmentlist, S.data(), sizeof(int) * S.size());
  return out->status = 0;
}

void gqm_cdt_free(gqm_cdt_result *r) {
  free(r->trianglelist);
  free(r->neighborlist);
  free(r->segmentlist);
  memset(r, 0, sizeof(*r));
}

}  // extern "C"
