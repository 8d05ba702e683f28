// C-ABI wrapper around the reference's vendored Triangle 1.6 (test oracle and
// CPU baseline only; never linked into the product).
//
// The reference builds its input CDTs with triangulate("pzQnc")
// (GPU_Refine/mesh.cpp:397) and times Triangle's CPU quality refinement with
// triangulate("pzDQnrq<theta>") for Ruppert mode or "pzQnrq<theta>" for Chew
// mode (GPU_Refine/main.cpp:389-407, CPU_Triangle_Quality).  These wrappers
// expose exactly those two calls to Python through plain pointers.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <sstream>
#include "triangle.h"

struct tri_result {
  int numberofpoints, numberoftriangles, numberofsegments;
  double *pointlist;
  int *trianglelist, *neighborlist, *segmentlist;
  double elapsed_ms;
};

static void take(triangulateio *o, tri_result *r) {
  r->numberofpoints = o->numberofpoints;
  r->numberoftriangles = o->numberoftriangles;
  r->numberofsegments = o->numberofsegments;
  r->pointlist = o->pointlist;
  r->trianglelist = o->trianglelist;
  r->neighborlist = o->neighborlist;
  r->segmentlist = o->segmentlist;
  // Triangle allocates with malloc (trimalloc); the fields below are not
  // handed out and are released here.
  free(o->pointmarkerlist);
  free(o->pointattributelist);
  free(o->triangleattributelist);
  free(o->segmentmarkerlist);
  free(o->edgelist);
  free(o->edgemarkerlist);
}

extern "C" {

// CDT of a PSLG as the reference builds its inputs (mesh.cpp:397, "pzQnc").
int tri_ref_cdt(int np, const double *pts, int ns, const int *segs, tri_result *r) {
  triangulateio in, out;
  memset(&in, 0, sizeof(in));
  memset(&out, 0, sizeof(out));
  in.numberofpoints = np;
  in.pointlist = const_cast<double *>(pts);
  in.numberofsegments = ns;
  in.segmentlist = const_cast<int *>(segs);
  char sw[] = "pzQnc";
  auto t0 = std::chrono::steady_clock::now();
  triangulate(sw, &in, &out, NULL);
  r->elapsed_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  take(&out, r);
  return 0;
}

// Triangle's CPU quality refinement on a CDT, as main.cpp:389-407 calls it.
int tri_ref_quality(int np, const double *pts, int nt, const int *tris, const int *nbrs, int ns, const int *segs,
                    double theta, int mode, tri_result *r) {
  triangulateio in, out;
  memset(&in, 0, sizeof(in));
  memset(&out, 0, sizeof(out));
  in.numberofpoints = np;
  in.pointlist = const_cast<double *>(pts);
  in.numberoftriangles = nt;
  in.numberofcorners = 3;
  in.trianglelist = const_cast<int *>(tris);
  in.neighborlist = const_cast<int *>(nbrs);
  in.numberofsegments = ns;
  in.segmentlist = const_cast<int *>(segs);
  std::ostringstream s;
  s << theta;
  std::string sw = (mode ? "pzDQnrq" : "pzQnrq") + s.str();
  auto t0 = std::chrono::steady_clock::now();
  triangulate(&sw[0], &in, &out, NULL);
  r->elapsed_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  take(&out, r);
  return 0;
}

void tri_ref_free(tri_result *r) {
  free(r->pointlist);
  free(r->trianglelist);
  free(r->neighborlist);
  free(r->segmentlist);
  memset(r, 0, sizeof(*r));
}
}
