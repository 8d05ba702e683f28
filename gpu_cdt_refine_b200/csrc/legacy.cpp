// GPU_Refine_Quality with the reference's signature (GPU_Refine/refine.h:385-386),
// forwarding to the C ABI.  Ownership and debug outputs follow
// GPU_Refine/refine.cu:7091-7125: new[] arrays owned by the caller.
#include <cstdio>
#include <cstring>

#include "../../include/gqm_refine.h"
#include "../../include/gqm_triangulateio.h"

void GPU_Refine_Quality(triangulateio *input, triangulateio *result, double theta, InsertPolicy insertpolicy,
                        DeletePolicy /*deletepolicy*/, int mode, int /*debug_iter*/, PStatus **ps_debug,
                        TStatus **ts_debug) {
  if (!result) return;
  result->numberofpoints = result->numberoftriangles = result->numberofsegments = 0;
  result->pointlist = nullptr;
  result->trianglelist = nullptr;
  result->neighborlist = nullptr;
  result->segmentlist = nullptr;
  if (!input) {
    fprintf(stderr, "GPU_Refine_Quality: %s\n", gqm_status_string(GQM_ERR_ARGUMENT));
    return;
  }
  gqm_cdt_in in;
  in.numberofpoints = input->numberofpoints;
  in.pointlist = input->pointlist;
  in.numberoftriangles = input->numberoftriangles;
  in.trianglelist = input->trianglelist;
  in.neighborlist = input->neighborlist;
  in.numberofsegments = input->numberofsegments;
  in.segmentlist = input->segmentlist;
  gqm_options opt;
  gqm_default_options(&opt);
  opt.theta = theta;
  opt.insert_policy = (insertpolicy == Offcenter) ? GQM_OFFCENTER : GQM_CIRCUMCENTER;
  opt.mode = mode ? GQM_RUPPERT : GQM_CHEW;
  gqm_cdt_out out;
  int rc = gqm_refine(&in, &out, &opt, nullptr);
  if (rc != GQM_OK) {
    fprintf(stderr, "GPU_Refine_Quality: %s (status %d)\n", gqm_status_string(rc), rc);
    return;
  }
  result->numberofpoints = out.numberofpoints;
  result->pointlist = new double[2 * (size_t)out.numberofpoints];
  memcpy(result->pointlist, out.pointlist, sizeof(double) * 2 * (size_t)out.numberofpoints);
  result->numberoftriangles = out.numberoftriangles;
  result->trianglelist = new int[3 * (size_t)out.numberoftriangles];
  memcpy(result->trianglelist, out.trianglelist, sizeof(int) * 3 * (size_t)out.numberoftriangles);
  result->neighborlist = new int[3 * (size_t)out.numberoftriangles];
  memcpy(result->neighborlist, out.neighborlist, sizeof(int) * 3 * (size_t)out.numberoftriangles);
  result->numberofsegments = out.numberofsegments;
  result->segmentlist = new int[2 * (size_t)out.numberofsegments];
  memcpy(result->segmentlist, out.segmentlist, sizeof(int) * 2 * (size_t)out.numberofsegments);
  if (ps_debug) {
    *ps_debug = new PStatus[out.numberofpoints];
    for (int i = 0; i < out.numberofpoints; ++i) (*ps_debug)[i]._status = out.pstatus[i];
  }
  if (ts_debug) {
    *ts_debug = new TStatus[out.numberoftriangles];
    for (int i = 0; i < out.numberoftriangles; ++i) (*ts_debug)[i]._status = out.tstatus[i];
  }
  gqm_free_result(&out);
}

// Release helpers for callers that cannot call delete[] themselves (ctypes):
// the arrays above are new[]-allocated exactly as in the reference.
extern "C" void gqm_legacy_free(triangulateio *r) {
  if (!r) return;
  delete[] r->pointlist;
  delete[] r->trianglelist;
  delete[] r->neighborlist;
  delete[] r->segmentlist;
  r->pointlist = nullptr;
  r->trianglelist = r->neighborlist = r->segmentlist = nullptr;
}
extern "C" void gqm_legacy_free_status(PStatus *ps, TStatus *ts) {
  delete[] ps;
  delete[] ts;
}
