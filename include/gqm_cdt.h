/* Constrained Delaunay triangulation of a planar straight-line graph: the
 * input construction step in front of the refiner.
 *
 * The refiner's input (GPU_Refine/refine.h:385-386) is a CDT in Triangle's
 * triangulateio layout built with the switches "pzQnc" (GPU_Refine/mesh.cpp:397):
 * zero-based indices, counterclockwise triangles, neighbour j opposite vertex j
 * (-1 on the boundary), and every convex hull edge a segment.  The reference
 * builds it with Triangle on the host (GPU_Refine/mesh.cpp:220-239); these
 * entry points build the same triangulation:
 *
 *   gqm_cdt_build      exact CPU builder (host library)
 *   gqm_cdt_build_gpu  the same contract on a CUDA device (device library)
 *
 * For points in general position (no four cocircular) the constrained
 * Delaunay triangulation is unique, so both return the same triangles up to
 * numbering; with cocircular points either may pick a different (equally
 * valid) diagonal.  Output segments: the input segments in input order (a
 * repeated pair kept once, at its first occurrence), then every hull edge that
 * is not an input segment.  Arrays are malloc'ed; release them with
 * gqm_cdt_free / gqm_cdt_gpu_free.
 */
#ifndef GQM_CDT_H
#define GQM_CDT_H

#include "gqm_refine.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gqm_cdt_result {
  int numberofpoints, numberoftriangles, numberofsegments, status;
  int *trianglelist, *neighborlist, *segmentlist;
} gqm_cdt_result;

/* status codes (shared by both builders) */
#define GQM_CDT_OK 0
#define GQM_CDT_ERR_FEW_POINTS (-1)      /* fewer than 3 points */
#define GQM_CDT_ERR_COLLINEAR (-2)       /* all points on one line */
#define GQM_CDT_ERR_SEGMENT (-4)         /* segment endpoint out of range, or a == b */
#define GQM_CDT_ERR_SEGMENTS_CROSS (-6)  /* two segments cross */
#define GQM_CDT_ERR_POINT_ON_SEGMENT (-7) /* a point lies in the interior of a segment */
#define GQM_CDT_ERR_DUPLICATE (-8)       /* two points with identical coordinates */
#define GQM_CDT_ERR_INTERNAL (-9)        /* an invariant failed (reported, never silent) */
#define GQM_CDT_ERR_CUDA (-10)
#define GQM_CDT_ERR_MEMORY (-11)
#define GQM_CDT_ERR_NO_DEVICE (-12)

typedef struct gqm_cdt_gpu_stats {
  int hull_vertices;      /* convex hull vertices, collinear ones included */
  int hull_candidates;    /* points left after the octagon filter */
  int insert_rounds;      /* point insertion rounds */
  int flip_rounds;        /* Lawson flip rounds (all phases) */
  int recover_rounds;     /* segment recovery rounds */
  int segments_missing;   /* segments not in the Delaunay triangulation of the points */
  long long flips;        /* Lawson flips */
  long long recover_flips; /* flips made while recovering segments */
  long long kernel_launches;
  double ms_h2d, ms_hull, ms_insert, ms_segments, ms_output, ms_d2h, ms_total;
} gqm_cdt_gpu_stats;

/* Host CPU builder (libgqm_host.so). */
int gqm_cdt_build(int np, const double *pts, int ns, const int *segs, gqm_cdt_result *out);
void gqm_cdt_free(gqm_cdt_result *r);

/* Device builder (libgqm_b200.so).  pts: np (x, y) pairs; segs: ns index
 * pairs; both host arrays.  stats may be NULL.  Returns a status code (also
 * stored in out->status); on failure out holds no arrays. */
int gqm_cdt_build_gpu(int np, const double *pts, int ns, const int *segs, int device, gqm_cdt_result *out,
                      gqm_cdt_gpu_stats *stats);
void gqm_cdt_gpu_free(gqm_cdt_result *r);
/* Status of this host thread's last device build (GQM_CDT_*). */
int gqm_cdt_gpu_last_status(void);
/* Frees the device buffers kept between calls on this host thread. */
void gqm_cdt_gpu_release(void);

/* Holes and regional attributes (host library; no counterpart in the
 * reference, which ignores both: Triangle's hole list and its `-A` regional
 * attributes, GPU_Refine/triangle.cpp).  A mesh whose arrays the library
 * malloc'ed; release it with gqm_mesh_free. */
typedef struct gqm_mesh {
  int numberofpoints;
  double *pointlist;
  int numberoftriangles;
  int *trianglelist;
  int *neighborlist;
  int numberofsegments;
  int *segmentlist;
} gqm_mesh;
/* The CDT (np points, nt triangles with neighbours, ns segments) without every
 * triangle reachable from one of the nholes hole points (x, y pairs) without
 * crossing a segment; vertices and segments no remaining triangle uses are
 * dropped, the rest renumbered in order.  Hole boundaries must be segments, so
 * the result is a valid refiner input.  GQM_OK, GQM_ERR_ARGUMENT (an index out
 * of range) or GQM_ERR_MEMORY. */
int gqm_remove_holes(int np, const double *pts, int nt, const int *tri, const int *nbr, int ns, const int *segs,
                     int nholes, const double *holes, gqm_mesh *out);
/* Regional attributes: regions holds nregions rows (x, y, attribute,
 * max_area), Triangle's regionlist layout.  Every triangle reachable from a
 * region's point without crossing a segment gets the region's attribute
 * (and max_area, when max_area is not NULL); regions are applied in order, a
 * later one overwriting an earlier one; unreached triangles get 0.  Regions
 * are bounded by segments and refinement keeps every segment, so on a refined
 * mesh this gives each triangle its input region's attribute. */
int gqm_region_attributes(int np, const double *pts, int nt, const int *tri, const int *nbr, int ns,
                          const int *segs, int nregions, const double *regions, double *attribute,
                          double *max_area);
void gqm_mesh_free(gqm_mesh *m);

/* The reference's whole flow in one call: Triangle "pzQnc" on the host
 * (GPU_Refine/mesh.cpp:397), then GPU_Refine_Quality (GPU_Refine/main.cpp:1862).  Here the CDT is built
 * on the device and refined there with no round trip through the host.
 * Returns a GQM_* status of gqm_refine; GQM_ERR_INPUT_CDT when the CDT could
 * not be built (gqm_cdt_gpu_last_status() then holds the builder's status).
 * The refined mesh is released with gqm_free_result; cdt_stats may be NULL. */
int gqm_triangulate_refine(int np, const double *pts, int ns, const int *segs, const gqm_options *opt,
                           gqm_cdt_out *out, gqm_stats *stats, gqm_cdt_gpu_stats *cdt_stats);

#ifdef __cplusplus
}
#endif

#endif
