/* gqm_triangulateio.h - C++ drop-in for the reference entry point.
 *
 * Declares GPU_Refine_Quality with the exact signature of
 * GPU_Refine/refine.h:385-386, so a program written against the reference
 * links against libgqm_b200.so unchanged (the mangled symbol is the same).
 * The types below are layout-compatible with the reference's:
 *   struct triangulateio  - Triangle 1.6 as vendored by the reference,
 *                           GPU_Refine/triangle.h:253-284 (including the
 *                           added numberofflips field);
 *   InsertPolicy, DeletePolicy - GPU_Refine/refine.h:32-33;
 *   PStatus, TStatus      - one status byte each, GPU_Refine/refine.h:36-205.
 * A program that already includes the reference's refine.h / triangle.h
 * should not include this header as well; the definitions are the same.
 *
 * Behaviour: as the reference, result->pointlist, trianglelist, neighborlist
 * and segmentlist are allocated with new[] and owned by the caller, and
 * *ps_debug / *ts_debug (when the pointers are non-NULL) receive new[] copies
 * of the compacted status arrays.  deletepolicy and debug_iter are accepted and
 * ignored, as in the reference.  Unlike the reference, a failure never exits
 * the process: it prints the status on stderr and returns a result with zero
 * points, triangles and segments.  gqm_refine() in gqm_refine.h returns the
 * status code instead.
 */
#ifndef GQM_TRIANGULATEIO_H
#define GQM_TRIANGULATEIO_H

#ifndef TRIANGLE_H_INCLUDED_BY_REFERENCE
struct triangulateio {
  double *pointlist;
  double *pointattributelist;
  int *pointmarkerlist;
  int numberofpoints;
  int numberofpointattributes;
  int *trianglelist;
  double *triangleattributelist;
  double *trianglearealist;
  int *neighborlist;
  int numberoftriangles;
  int numberofcorners;
  int numberoftriangleattributes;
  int *segmentlist;
  int *segmentmarkerlist;
  int numberofsegments;
  double *holelist;
  int numberofholes;
  double *regionlist;
  int numberofregions;
  int *edgelist;
  int *edgemarkerlist;
  double *normlist;
  int numberofedges;
  int numberofflips;
};
#endif

#ifdef __cplusplus
typedef enum { Circumcenter, Offcenter } InsertPolicy;
typedef enum { Strict, Connected, Orthogonal, noDeletion, DeleteFromDT, noPriority } DeletePolicy;
typedef struct PStatus {
  unsigned char _status;
} PStatus;
typedef struct TStatus {
  unsigned char _status;
} TStatus;

void GPU_Refine_Quality(triangulateio *input, triangulateio *result, double theta, InsertPolicy insertpolicy,
                        DeletePolicy deletepolicy, int mode, int debug_iter, PStatus **ps_debug, TStatus **ts_debug);
#endif

#endif
