// GPU_Refine_Quality with the reference's signature (GPU_Refine/refine.h:385-386),
// forwarding to the C ABI.  Ownership and debug outputs follow
// GPU_Refine/refine.cu:7091-7125: new[] arrays owned by the caller.
#include <cstdio>
#include <cstring>

#include "../../include/gqm_refine.h"
#include "../../include/gqm_triangulateio.h"
#include "host_copy.h"

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
  // new[] arrays as the reference hands them out, filled on the host's cores
  const size_t np = (size_t)out.numberofpoints, nt = (size_t)out.numberoftriangles, ns = (size_t)out.numberofsegments;
  result->numberofpoints = out.numberofpoints;
  result->pointlist = new double[2 * np];
  result->numberoftriangles = out.numberoftriangles;
  result->trianglelist = new int[3 * nt];
  result->neighborlist = new int[3 * nt];
  result->numberofsegments = out.numberofsegments;
  result->segmentlist = new int[2 * ns];
  advise_huge(result->pointlist, 16 * np);
  advise_huge(result->trianglelist, 12 * nt);
  advise_huge(result->neighborlist, 12 * nt);
  host_copy({{result->pointlist, out.pointlist, 16 * np}, {result->trianglelist, out.trianglelist, 12 * nt},
             {result->neighborlist, out.neighborlist, 12 * nt}, {result->segmentlist, out.segmentlist, 8 * ns}});
  static_assert(sizeof(PStatus) == 1 && sizeof(TStatus) == 1, "one status byte per point and triangle");
  if (ps_debug) {
    *ps_debug = new PStatus[np];
    memcpy(*ps_debug, out.pstatus, np);
  }
  if (ts_debug) {
    *ts_debug = new TStatus[nt];
    memcpy(*ts_debug, out.tstatus, nt);
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
