// Holes and regional attributes of a constrained Delaunay triangulation
// (host library).  The reference ignores both (its input contract is a CDT
// without holes, GPU_Refine/refine.h:385-386); Triangle, whose switches the
// reference's callers use (GPU_Refine/mesh.cpp:397), provides them through its
// hole list and its regional attribute list (triangle.cpp's `-A` switch,
// spread by its region flood fill).  Here:
//
//  * gqm_remove_holes: every triangle reachable from a hole point without
//    crossing a segment is removed, vertices and segments no remaining
//    triangle uses are dropped and the rest renumbered (kept in their order).
//    Hole boundaries must be segments, so the result is a valid refiner input
//    (every boundary edge a segment).
//  * gqm_region_attributes: every triangle reachable from a region point
//    without crossing a segment takes that region's attribute (and its area
//    bound); regions are applied in order, a later one overwriting an earlier
//    one; triangles that no region reaches get attribute 0 and no bound.
//    Regions are bounded by segments and refinement never removes a segment,
//    so applying it to the refined mesh gives every output triangle the
//    attribute of the input region it lies in.
//
// A point is located by a scan of the triangles with exact orientation tests
// (a point on an edge belongs to the first triangle found).  Flood fills are
// breadth-first over neighbour links whose edge is not a segment.
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <unordered_set>
#include <vector>

#include "../../include/gqm_cdt.h"
#include "predicates.h"

namespace {

inline uint64_t edge_key(int a, int b) {
  const uint32_t lo = (uint32_t)std::min(a, b), hi = (uint32_t)std::max(a, b);
  return ((uint64_t)hi << 32) | lo;
}

struct View {
  int np, nt, ns;
  const double *pts;
  const int *tri, *nbr, *segs;
};

int check(const View &v) {
  if (v.np < 3 || v.nt < 1 || v.ns < 0 || !v.pts || !v.tri || !v.nbr || (v.ns > 0 && !v.segs))
    return GQM_ERR_ARGUMENT;
  for (long i = 0; i < 3L * v.nt; ++i)
    if (v.tri[i] < 0 || v.tri[i] >= v.np || v.nbr[i] < -1 || v.nbr[i] >= v.nt) return GQM_ERR_ARGUMENT;
  for (long i = 0; i < 2L * v.ns; ++i)
    if (v.segs[i] < 0 || v.segs[i] >= v.np) return GQM_ERR_ARGUMENT;
  return GQM_OK;
}

// triangle containing (x, y), or -1
int locate(const View &v, double x, double y) {
  for (int t = 0; t < v.nt; ++t) {
    const int a = v.tri[3 * t], b = v.tri[3 * t + 1], c = v.tri[3 * t + 2];
    const double *pa = v.pts + 2 * a, *pb = v.pts + 2 * b, *pc = v.pts + 2 * c;
    if (gqm_orient_exact(pa[0], pa[1], pb[0], pb[1], x, y) >= 0 &&
        gqm_orient_exact(pb[0], pb[1], pc[0], pc[1], x, y) >= 0 &&
        gqm_orient_exact(pc[0], pc[1], pa[0], pa[1], x, y) >= 0)
      return t;
  }
  return -1;
}

// triangles reachable from `start` without crossing a segment, marked `mark`
// in label[] (entries equal to `mark` already are not revisited)
void flood(const View &v, const std::unordered_set<uint64_t> &segset, int start, std::vector<int> &label,
           int mark, std::vector<int> &stack) {
  stack.clear();
  stack.push_back(start);
  label[start] = mark;
  while (!stack.empty()) {
    const int t = stack.back();
    stack.pop_back();
    for (int j = 0; j < 3; ++j) {
      const int n = v.nbr[3 * t + j];
      if (n < 0 || label[n] == mark) continue;
      if (segset.count(edge_key(v.tri[3 * t + (j + 1) % 3], v.tri[3 * t + (j + 2) % 3]))) continue;
      label[n] = mark;
      stack.push_back(n);
    }
  }
}

std::unordered_set<uint64_t> segment_set(const View &v) {
  std::unordered_set<uint64_t> s;
  s.reserve(2 * (size_t)v.ns + 8);
  for (int i = 0; i < v.ns; ++i) s.insert(edge_key(v.segs[2 * i], v.segs[2 * i + 1]));
  return s;
}

}  // namespace

extern "C" {

int gqm_remove_holes(int np, const double *pts, int nt, const int *tri, const int *nbr, int ns, const int *segs,
                     int nholes, const double *holes, gqm_mesh *out) {
  if (!out || nholes < 0 || (nholes > 0 && !holes)) return GQM_ERR_ARGUMENT;
  memset(out, 0, sizeof(*out));
  const View v{np, nt, ns, pts, tri, nbr, segs};
  int rc = check(v);
  if (rc) return rc;
  const std::unordered_set<uint64_t> segset = segment_set(v);
  std::vector<int> drop(nt, 0), stack;
  for (int h = 0; h < nholes; ++h) {
    const int t = locate(v, holes[2 * h], holes[2 * h + 1]);
    if (t >= 0 && !drop[t]) flood(v, segset, t, drop, 1, stack);
  }
  std::vector<int> newt(nt, -1), newp(np, -1);
  int kt = 0, kp = 0;
  for (int t = 0; t < nt; ++t)
    if (!drop[t]) newt[t] = kt++;
  std::vector<char> used(np, 0);
  std::unordered_set<uint64_t> kept_edges;
  kept_edges.reserve(3 * (size_t)kt + 8);
  for (int t = 0; t < nt; ++t)
    if (!drop[t])
      for (int j = 0; j < 3; ++j) {
        used[tri[3 * t + j]] = 1;
        kept_edges.insert(edge_key(tri[3 * t + (j + 1) % 3], tri[3 * t + (j + 2) % 3]));
      }
  for (int i = 0; i < np; ++i)
    if (used[i]) newp[i] = kp++;
  int ks = 0;
  for (int s = 0; s < ns; ++s) ks += kept_edges.count(edge_key(segs[2 * s], segs[2 * s + 1])) ? 1 : 0;
  out->pointlist = (double *)malloc(sizeof(double) * 2 * (size_t)std::max(kp, 1));
  out->trianglelist = (int *)malloc(sizeof(int) * 3 * (size_t)std::max(kt, 1));
  out->neighborlist = (int *)malloc(sizeof(int) * 3 * (size_t)std::max(kt, 1));
  out->segmentlist = (int *)malloc(sizeof(int) * 2 * (size_t)std::max(ks, 1));
  if (!out->pointlist || !out->trianglelist || !out->neighborlist || !out->segmentlist) {
    gqm_mesh_free(out);
    return GQM_ERR_MEMORY;
  }
  for (int i = 0; i < np; ++i)
    if (newp[i] >= 0) {
      out->pointlist[2 * newp[i]] = pts[2 * i];
      out->pointlist[2 * newp[i] + 1] = pts[2 * i + 1];
    }
  for (int t = 0; t < nt; ++t) {
    const int k = newt[t];
    if (k < 0) continue;
    for (int j = 0; j < 3; ++j) {
      out->trianglelist[3 * k + j] = newp[tri[3 * t + j]];
      const int n = nbr[3 * t + j];
      out->neighborlist[3 * k + j] = n >= 0 ? newt[n] : -1;
    }
  }
  ks = 0;
  for (int s = 0; s < ns; ++s)
    if (kept_edges.count(edge_key(segs[2 * s], segs[2 * s + 1]))) {
      out->segmentlist[2 * ks] = newp[segs[2 * s]];
      out->segmentlist[2 * ks + 1] = newp[segs[2 * s + 1]];
      ks++;
    }
  out->numberofpoints = kp;
  out->numberoftriangles = kt;
  out->numberofsegments = ks;
  return GQM_OK;
}

int gqm_region_attributes(int np, const double *pts, int nt, const int *tri, const int *nbr, int ns,
                          const int *segs, int nregions, const double *regions, double *attribute,
                          double *max_area) {
  if (nregions < 0 || (nregions > 0 && !regions) || !attribute) return GQM_ERR_ARGUMENT;
  const View v{np, nt, ns, pts, tri, nbr, segs};
  int rc = check(v);
  if (rc) return rc;
  const std::unordered_set<uint64_t> segset = segment_set(v);
  std::vector<int> label(nt, -1), stack;
  for (int r = 0; r < nregions; ++r) {
    const int t = locate(v, regions[4 * r], regions[4 * r + 1]);
    if (t >= 0) flood(v, segset, t, label, r, stack);
  }
  for (int t = 0; t < nt; ++t) {
    attribute[t] = label[t] >= 0 ? regions[4 * label[t] + 2] : 0.0;
    if (max_area) max_area[t] = label[t] >= 0 ? regions[4 * label[t] + 3] : 0.0;
  }
  return GQM_OK;
}

void gqm_mesh_free(gqm_mesh *m) {
  if (!m) return;
  free(m->pointlist);
  free(m->trianglelist);
  free(m->neighborlist);
  free(m->segmentlist);
  memset(m, 0, sizeof(*m));
}

}  // extern "C"
