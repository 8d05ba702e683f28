/* Test oracle: CPU restatement of the reference's GPU quality refinement.
 *
 * This header and gqm_oracle.c are test infrastructure.  Only the tests, the
 * smoke check and the CPU-baseline leg of bench.py use them, as the checker;
 * the product never calls them.
 *
 * gqm_oracle_refine() follows GPU_Refine_Quality (GPU_Refine/refine.cu:6500-7139)
 * step by step.  Every GPU kernel is emulated by running its thread body for
 * each thread position in ascending order over the state the previous kernel
 * left.  Where the reference's threads race (see gqm_oracle.c for the list),
 * a fixed rule is used that the CUDA implementation shares.
 */
#ifndef GQM_ORACLE_H
#define GQM_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int numberofpoints, numberoftriangles, numberofsegments;
  double *pointlist;     /* 2 * numberofpoints */
  int *trianglelist;     /* 3 * numberoftriangles, plain neighbour format below */
  int *neighborlist;     /* 3 * numberoftriangles */
  int *segmentlist;      /* 2 * numberofsegments */
  unsigned char *pstatus; /* PStatus bytes of the compacted points */
  unsigned char *tstatus; /* TStatus bytes of the compacted triangles */
  int rounds;            /* iterations of the quality loop */
  int status;            /* 0 ok, <0 error */
  long long flip_steps, steiner_inserted, midpoints_inserted, bad_total;
} gqm_oracle_out;

/* policy: 0 Circumcenter, 1 Offcenter.  mode: 1 Ruppert, 0 Chew.
 * max_rounds bounds every loop (0 = no bound); exceeding it returns -2.
 * nbr uses Triangle's plain format (neighbour triangle index, -1 boundary). */
int gqm_oracle_refine(int np, const double *pts, int nt, const int *tri, const int *nbr, int ns, const int *segs,
                      double theta, int policy, int mode, long long max_rounds, gqm_oracle_out *out);
/* Same, with cos^2(theta) given.  The reference evaluates cos(theta*PI/180)
 * on the device (refine.cu:418-419), whose cos() can differ from the host's
 * by one ulp for some angles (it does at 20.7 degrees); goodcos2 > 0 replaces
 * the host evaluation by that device value.  goodcos2 <= 0: host cos(). */
int gqm_oracle_refine_gc(int np, const double *pts, int nt, const int *tri, const int *nbr, int ns,
                         const int *segs, double theta, double goodcos2, int policy, int mode, long long max_rounds,
                         gqm_oracle_out *out);
void gqm_oracle_free(gqm_oracle_out *out);

/* Area bound of the following refinements (0: none): a triangle larger than
 * `a` is refined whatever its angles (Triangle's `a` switch). */
void gqm_oracle_set_max_area(double a);

/* Debugging aid: write one digest line per flip step to `path` (NULL: off). */
void gqm_oracle_trace(const char *path);
void gqm_oracle_trace_dump(long step, const char *path);

/* Reference predicate arithmetic, exported for the predicate tests. */
double gqm_oracle_orient(const double *a, const double *b, const double *c);
double gqm_oracle_incircle(const double *a, const double *b, const double *c, const double *d);
double gqm_oracle_incircle_exact(const double *a, const double *b, const double *c, const double *d);
void gqm_oracle_circumcenter(const double *apex, const double *org, const double *dest, double offconstant,
                             int offcenter, double *out);

#ifdef __cplusplus
}
#endif
#endif
