/* gqm_refine.h - C ABI of the B200 constrained-Delaunay quality refiner.
 *
 * Every entry point takes plain pointers and sizes and returns a status code
 * (GQM_OK == 0, negative on error); none of them exits the process.
 *
 * Reference interface replaced (chenzhenghai/GPU_CDT_Refine):
 *   void GPU_Refine_Quality(triangulateio *input, triangulateio *result,
 *        double theta, InsertPolicy insertpolicy, DeletePolicy deletepolicy,
 *        int mode, int debug_iter, PStatus **ps_debug, TStatus **ts_debug);
 *   declared at GPU_Refine/refine.h:385-386, defined at
 *   GPU_Refine/refine.cu:6500-7139.
 * The C++ drop-in with that exact signature is in gqm_triangulateio.h and
 * forwards to gqm_refine() below.
 */
#ifndef GQM_REFINE_H
#define GQM_REFINE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define GQM_OK 0
#define GQM_ERR_ARGUMENT (-1)     /* null pointer or inconsistent sizes */
#define GQM_ERR_ROUND_LIMIT (-2)  /* a refinement loop exceeded options.max_rounds */
#define GQM_ERR_WALK_LIMIT (-3)   /* a point-location walk did not end */
#define GQM_ERR_FAN_LIMIT (-4)    /* a vertex fan walk did not close */
#define GQM_ERR_TOPOLOGY (-5)     /* mesh inconsistency found on the device */
#define GQM_ERR_CAVITY (-6)       /* cavity walk exceeded its bound */
#define GQM_ERR_CUDA (-10)        /* a CUDA runtime call failed */
#define GQM_ERR_NO_DEVICE (-11)   /* no CUDA device */
#define GQM_ERR_MEMORY (-12)      /* device allocation failed */
#define GQM_ERR_ARENA (-14)       /* a batched domain outgrew its block's scratch arena */
#define GQM_ERR_INPUT_CDT (-15)   /* gqm_triangulate_refine: the CDT could not be built (gqm_cdt_gpu_last_status) */

/* InsertPolicy (GPU_Refine/refine.h:32) */
#define GQM_CIRCUMCENTER 0
#define GQM_OFFCENTER 1
/* refinement mode (GPU_Refine/refine.cu:131: run_mode != 0 is Ruppert) */
#define GQM_CHEW 0
#define GQM_RUPPERT 1
/* Steiner placement (no counterpart in the reference beyond the plain rule) */
#define GQM_PLACE_PLAIN 0   /* off-center / circumcenter as GPU_Refine/refine.cu:3780-3868 */
#define GQM_PLACE_LEARNED 1 /* a point between the off-center and the circumcenter chosen by a small
                               network, with the plain off-center as the fallback (see below) */
/* predicate arithmetic */
#define GQM_PRED_REFERENCE 0 /* the reference's effective FP64 arithmetic (bit-exact parity) */
#define GQM_PRED_EXACT 1     /* exact orient2d/incircle (adaptive filter + expansions) */

/* Input CDT in Triangle's triangulateio layout (GPU_Refine/triangle.h:253-284):
 * zero-based indices, counterclockwise triangles, neighbour j opposite vertex
 * j (-1 on the boundary), convex hull enclosed by segments. */
typedef struct {
  int numberofpoints;
  const double *pointlist;   /* 2 * numberofpoints, x y interleaved */
  int numberoftriangles;
  const int *trianglelist;   /* 3 * numberoftriangles */
  const int *neighborlist;   /* 3 * numberoftriangles */
  int numberofsegments;
  const int *segmentlist;    /* 2 * numberofsegments */
} gqm_cdt_in;

/* Output CDT.  Arrays are allocated by the library and released with
 * gqm_free_result() (never free() them one by one): a result of 16 MB or more
 * lives in one block of pinned host memory that the library downloads into
 * directly and reuses for a later result once it is released (the domains of
 * a persistent batch share one block, free again once every domain's result is
 * released; at most 8 GB of such blocks); a smaller one is malloc()ed.  pstatus / tstatus hold the
 * reference's PStatus / TStatus bytes of the compacted points / triangles
 * (refine.h:36-205). */
typedef struct {
  int numberofpoints;
  double *pointlist;
  int numberoftriangles;
  int *trianglelist;
  int *neighborlist;
  int numberofsegments;
  int *segmentlist;
  unsigned char *pstatus;
  unsigned char *tstatus;
} gqm_cdt_out;

typedef struct {
  double theta;         /* minimum angle in degrees */
  int insert_policy;    /* GQM_CIRCUMCENTER / GQM_OFFCENTER */
  int mode;             /* GQM_RUPPERT / GQM_CHEW */
  int predicates;       /* GQM_PRED_REFERENCE / GQM_PRED_EXACT */
  int device;           /* CUDA device ordinal */
  long long max_rounds; /* bound on every refinement loop; 0 = default (1e6) */
  int placement;        /* GQM_PLACE_PLAIN (the reference's rule) / GQM_PLACE_LEARNED */
  const float *mlp;     /* GQM_PLACE_LEARNED: host array of GQM_MLP_PARAMS network parameters */
  double max_area;      /* area bound (no counterpart in the reference; Triangle's `a` switch):
                           triangles larger than this are refined whatever their angles; 0 = none */
} gqm_options;

typedef struct {
  int rounds;                   /* quality iterations */
  long long flip_steps;         /* flip-flop steps */
  long long steiner_inserted;   /* interior/edge Steiner points inserted */
  long long midpoints_inserted; /* subsegment split points inserted */
  long long bad_total;          /* bad triangles summed over rounds */
  long long host_syncs;         /* device-to-host count reads */
  long long kernel_launches;    /* kernels run by the refinement, those inside the flip-loop graphs included */
  long long exact_fallbacks;    /* incircle tests that needed the expansion path (single-domain
                                   path; a device-wide count, so concurrent runs on one device add up) */
  double goodcos2;              /* cos^2(theta) as evaluated on the device */
  double device_ms;             /* device time of the refinement (CUDA events) */
  long long learned_candidates; /* GQM_PLACE_LEARNED: Steiner points where the rule could apply */
  long long learned_used;       /* ... of which the network's point was inserted */
} gqm_stats;

/* Default options: theta 20, Offcenter, Ruppert, reference predicates, device 0. */
void gqm_default_options(gqm_options *opt);

/* One call: host CDT in, host CDT out (host<->device copies included).
 * Equivalent of GPU_Refine_Quality.  Device buffers are kept in one cached
 * context per device between calls; calls are serialized by a mutex. */
int gqm_refine(const gqm_cdt_in *in, gqm_cdt_out *out, const gqm_options *opt, gqm_stats *stats);
void gqm_free_result(gqm_cdt_out *out);

/* Reusable context: device buffers are kept between runs. */
typedef struct gqm_context gqm_context;
int gqm_context_create(int device, gqm_context **ctx);
void gqm_context_destroy(gqm_context *ctx);
/* Refine a CDT whose arrays already reside in device memory (in_on_device != 0)
 * or in host memory; the result stays on the device until gqm_context_result. */
int gqm_context_run(gqm_context *ctx, const gqm_cdt_in *in, int in_on_device, const gqm_options *opt,
                    gqm_stats *stats);
int gqm_context_result(gqm_context *ctx, gqm_cdt_out *out);
/* Sizes of the last result without copying it. */
int gqm_context_result_sizes(gqm_context *ctx, int *npoints, int *ntriangles, int *nsegments);
/* Measurement probe (no counterpart in the reference).  While enabled, the
 * two kernels that take most of the device time, the grid-wide flip-step check
 * kernel and the small-step kernel (whole flip steps of small active sets in
 * one launch), timestamp every launch on the device: from its first block's
 * start to its last block's end (%globaltimer); the flip-flop loops are timed
 * on the device as well, from entry to their last step.  gqm_context_probe(ctx, 1)
 * resets and enables, (ctx, 0) disables; gqm_context_probe_read sums since the
 * reset. */
typedef struct {
  long long check_launches; /* launches of the flip-step check kernel */
  long long check_items;    /* active triangles they checked */
  double check_ms;          /* their summed execution time */
  long long loop_launches;  /* flip-flop loops run */
  double loop_ms;           /* their summed device time (%globaltimer at loop entry and end) */
  long long first_items[4]; /* active triangles of the first four check launches */
  long long small_launches; /* launches of the small-step kernel */
  long long small_items;    /* active triangles of the flip steps they ran */
  long long small_winners;  /* flips and flops those steps applied */
  double small_ms;          /* their summed execution time */
} gqm_probe;
int gqm_context_probe(gqm_context *ctx, int enable);
int gqm_context_probe_read(gqm_context *ctx, gqm_probe *p);

/* Flip-step profile of the last run (no counterpart in the reference):
 * steps[b] = flip steps whose active set held [2^b, 2^(b+1)) triangles,
 * items[b] = those steps' active triangles summed; 32 bins each. */
int gqm_context_flip_profile(gqm_context *ctx, long long *steps, long long *items);
/* The CUDA stream the context launches on (a cudaStream_t). */
void *gqm_context_stream(gqm_context *ctx);

/* Launch shape of a context's flip-flop loop.  Replaces the reference's fixed
 * BLOCK_SIZE (GPU_Refine/refine.h:19) and its per-kernel grid sizes
 * (maxnumofblock, GPU_Refine/refine.cu:5223,5238,6538) for the loop that takes
 * most of the device time (flipFlop, refine.cu:2328-2490).  No field changes a
 * result: every flip step makes the reference's decisions whatever the launch
 * shape.  Zero in a field means its default. */
typedef struct {
  int step_grid;           /* blocks of 256 threads of each grid-wide flip-step kernel (default 592, 4 per SM) */
  int small_limit;         /* flip steps of at most this many active triangles run inside one launch of the
                              small-step kernel (default 1024; negative: never) */
  int small_cluster;       /* small-step kernel: 1 = one block of 512 threads (default); 8 or 16 = one
                              thread-block cluster of that many 256-thread blocks */
  int check_blocks_per_sm; /* register budget of the flip-step check kernel: 2 resident 256-thread blocks
                              per SM (default; at most 128 registers) or 1 (up to 255) */
} gqm_tuning;
/* Set / read a context's launch shape.  Set returns GQM_ERR_ARGUMENT for a
 * value out of range and GQM_ERR_CUDA when the device cannot run the requested
 * cluster size; the context keeps its previous shape then. */
int gqm_context_set_tuning(gqm_context *ctx, const gqm_tuning *t);
int gqm_context_get_tuning(gqm_context *ctx, gqm_tuning *t);
/* Autotuner (no counterpart in the reference): refines `in` (host or device
 * arrays, as gqm_context_run) once per candidate launch shape, one field at a
 * time (check kernel budget, small-step kernel, small-step limit, step grid),
 * keeping each field's fastest value by the device time of the refinement
 * (the best of `repeats` runs, at least 1).  The chosen shape is set on the
 * context and written to *chosen; *best_ms (may be NULL) receives its time.
 * `in` is typically a sample of the workload to be refined; its result is
 * left in the context like any run's. */
int gqm_context_autotune(gqm_context *ctx, const gqm_cdt_in *in, int in_on_device, const gqm_options *opt,
                         int repeats, gqm_tuning *chosen, double *best_ms);
/* Launch shape of the context that gqm_refine keeps for `device` (created by
 * this call when it does not exist yet), e.g. a shape gqm_context_autotune
 * chose on a sample of the caller's workload. */
int gqm_set_default_tuning(int device, const gqm_tuning *t);

/* Copy the last result of `ctx` into arrays the caller already owns, without
 * allocating any memory, host or device.
 *
 * No counterpart in the reference: its result path always allocates (new[] on
 * the host, device_vector on the GPU).  gqm_context_result() above also
 * allocates: it mallocs the host arrays on every call, and it grows its device
 * and pinned staging buffers (cudaMalloc, and a cudaFree that synchronizes the
 * whole device) whenever a result larger than any before arrives.  Callers that
 * cannot do that - a service that fixes its device memory budget at start-up
 * and reads many small results in a steady-state loop, or code sharing the GPU
 * with work that must not be stalled by an implicit device-wide sync - use
 * this entry point instead.
 *
 * The caller fills out->pointlist, trianglelist, neighborlist, segmentlist,
 * pstatus and tstatus with buffers sized from gqm_context_result_sizes(); the
 * counts are written back.  Staging goes through one statically allocated
 * device array of GQM_NOALLOC_MAX_ELEMENTS rows (about 4.4 MB), which every GPU
 * that loads the library holds until the process exits.  A result with more
 * points, triangles or segments than GQM_NOALLOC_MAX_ELEMENTS is rejected with
 * GQM_ERR_TOO_LARGE.  The first call on a device looks up that array's device
 * address (cudaGetSymbolAddress); make that first call before any stream
 * capture.  All calls on one device share the array, so calls that overlap on
 * the GPU (from different host threads or contexts) race; serialize them. */
#define GQM_NOALLOC_MAX_ELEMENTS 131072
#define GQM_ERR_TOO_LARGE (-13)
int gqm_context_result_noalloc(gqm_context *ctx, gqm_cdt_out *out);

/* Batched refinement of independent domains (no counterpart in the
 * reference, which refines one CDT per call).  Domains are taken largest first
 * by `workers` host threads; each worker owns a context with its own CUDA
 * stream, so the GPU work of different domains overlaps.  opt[i] and stats[i]
 * belong to domain i (stats may be NULL); out[i] is released with
 * gqm_free_result.  Each domain's result is the one gqm_refine would return.
 * Returns GQM_OK or the first failing domain's status (*failed_domain set). */
int gqm_refine_batch(int ndomains, const gqm_cdt_in *in, gqm_cdt_out *out, const gqm_options *opt,
                     gqm_stats *stats, int workers, int *failed_domain);

/* Persistent batched refinement (no counterpart in the reference, which
 * refines one CDT per call).  One kernel launch refines every domain: each
 * thread block takes the next domain from a queue ordered largest first and
 * runs the whole refinement of it (rounds, flip-flop loops, compaction) on the
 * device, in a scratch arena of its own sized for the largest domain.  Each
 * domain's result is the one gqm_refine would return for it.  A domain whose
 * mesh outgrows its arena (GQM_ERR_ARENA) is refined again by the
 * single-domain GPU path; report->fallbacks counts those.  All domains must
 * name the same device.  Device and pinned host buffers are kept per device
 * between calls (grow only) and released by gqm_batch_release. */
typedef struct {
  int threads_per_block; /* 128, 256 or 512; 0 = the autotuned choice */
  int blocks_per_sm;     /* resident blocks per SM asked of the compiler; 0 = autotuned */
  double memory_fraction;/* share of the free device memory the call may take; 0 = 0.8 */
} gqm_batch_options;
typedef struct {
  int grid;              /* blocks launched */
  int threads_per_block;
  int blocks_per_sm;
  int fallbacks;         /* domains re-run by the single-domain path */
  long long arena_bytes; /* scratch arena of one block */
  double kernel_ms;      /* the persistent launches (CUDA events) */
  double h2d_ms, d2h_ms; /* input upload; output download and unpacking */
  double total_ms;       /* the whole call */
} gqm_batch_report;
void gqm_default_batch_options(gqm_batch_options *b);
int gqm_refine_batch_persistent(int ndomains, const gqm_cdt_in *in, gqm_cdt_out *out, const gqm_options *opt,
                                gqm_stats *stats, const gqm_batch_options *bopt, gqm_batch_report *report,
                                int *failed_domain);
/* Autotuner of the persistent batch: times every compiled (threads per block,
 * blocks per SM) variant on the given sample of domains, keeps the fastest as
 * the autotuned choice of that device for later calls, and returns it in
 * *chosen (and each variant's kernel time in ms_per_variant[k], k < the value
 * returned by gqm_batch_variants, when not NULL). */
int gqm_batch_variants(int *threads, int *blocks_per_sm, int max);
int gqm_batch_autotune(int ndomains, const gqm_cdt_in *in, const gqm_options *opt, gqm_batch_options *chosen,
                       double *ms_per_variant);
void gqm_batch_release(int device);

/* Learned Steiner placement (no counterpart in the reference).  Where the
 * reference inserts an off-center (a point on the bisector of the bad
 * triangle's shortest edge, nearer than the circumcenter), GQM_PLACE_LEARNED
 * inserts the point at  s_off + t (s_cc - s_off)  on that bisector instead,
 * t = the network's output for the triangle's 32 features; the off-center is
 * kept when t <= 0 or t >= 1 or when the point would encroach a subsegment of
 * the triangle or its neighbours.  The network is 32 -> 64 -> 64 -> 1 with
 * ReLU, bf16 weights and fp32 accumulation on the tensor cores.  Parameters
 * are GQM_MLP_PARAMS floats: W1[64][32], b1[64], W2[64][64], b2[64], w3[64],
 * b3 (weights are rounded to bf16 on the device). */
#define GQM_MLP_FEATURES 32
#define GQM_MLP_PARAMS 6337
/* Training data from a plain refinement of `in` (opt->placement is ignored):
 * for every bad triangle where the learned rule applies, its features
 * (GQM_MLP_FEATURES floats) and a target t in [0, 1]: of nine points
 * t = 0, 1/8, ..., 1 on the bisector, the one whose new triangles (the point
 * joined to its Delaunay cavity's boundary) include the fewest with an angle
 * below theta, ties to the smaller t (the off-center unless a point beyond it
 * is strictly better); points that encroach a subsegment are excluded.  Up to `cap` rows; *count gets the number written. */
int gqm_learn_collect(const gqm_cdt_in *in, const gqm_options *opt, float *features, float *targets,
                      long long cap, long long *count);
/* Exploration run for descendant-count labels (opt->placement is ignored).
 * Every bad triangle the refinement splits gets one row, in the order the
 * rounds reach them; the candidate's point is placed at
 * t = j / (levels - 1) of the way from the off-center to the circumcenter,
 * j drawn per triangle from a hash of `seed` and its vertex ids (the
 * off-center when that point would encroach a subsegment of the triangle or
 * its neighbours).  Per row: the triangle's features (GQM_MLP_FEATURES floats,
 * all zero where off-center and circumcenter coincide), level[] = j (-1 for
 * those), t_used[] = the t inserted, parent[] = the row that inserted the
 * youngest vertex of the bad triangle (-1: all its vertices are input
 * vertices or descend from none), inserted[] = 1 when the point entered the
 * mesh (a candidate that lost its conflict has 0 and a later row for the same
 * triangle), midpoints[] = subsegment midpoints whose youngest neighbouring
 * vertex the row inserted.  The descendants of a row are the rows and
 * midpoints below it in the parent tree.  With a network `mlp` (GQM_MLP_PARAMS
 * floats, else NULL), a triangle draws a level only with probability `eps`
 * (from the same hash) and otherwise takes the network's t as the learned rule
 * would, with level[] = -2.  *count gets the number of rows; more than `cap`
 * rows returns GQM_ERR_TOO_LARGE with no rows written (2..64 levels,
 * 0 <= eps <= 1, cap <= INT_MAX). */
int gqm_learn_explore(const gqm_cdt_in *in, const gqm_options *opt, int levels, unsigned seed, const float *mlp,
                      float eps, float *features, int *level, float *t_used, int *parent, unsigned char *inserted,
                      int *midpoints, long long cap, long long *count);
/* Network output (the unclamped t) for n feature rows. */
int gqm_mlp_infer(int device, const float *params, const float *features, long long n, float *out);
/* Mean squared error of the network on n rows and its gradient with respect
 * to every parameter (the GPU forward and backward kernels). */
int gqm_mlp_grad(int device, const float *params, const float *features, const float *targets, long long n,
                 float *loss, float *grad);
/* Adam training of params (in place) on n rows: `epochs` passes in
 * mini-batches of `batch` rows (a multiple of 64), learning rate lr, rows
 * shuffled with `seed`; *loss gets the last epoch's mean loss. */
int gqm_mlp_train(int device, float *params, const float *features, const float *targets, long long n,
                  int epochs, int batch, float lr, unsigned seed, float *loss);
/* Device time of the network alone: the inference kernel over n rows of
 * zero features (the work does not depend on the values), timed with CUDA
 * events over `iters` launches after one untimed launch; *ms gets the mean
 * per launch. */
int gqm_mlp_time(int device, const float *params, long long n, int iters, float *ms);

const char *gqm_status_string(int status);
int gqm_version(void);

/* Floating-point arithmetic the library's refiner kernels were compiled with.
 * GQM_ARITH_SEPARATE (libgqm_b200.so): every product and sum rounded on its
 * own (nvcc -fmad=false), the arithmetic of the reference built with
 * -fmad=false, which the CPU oracle restates.  GQM_ARITH_CONTRACTED
 * (libgqm_b200_fma.so): nvcc's default contraction of a product feeding an
 * add or subtract into one fused multiply-add, the arithmetic of the reference
 * as its project builds it (GPU_Refine/GPU_Refine.vcxproj sets no -fmad
 * option).  The two give different meshes wherever a rounding decides a
 * predicate or moves a Steiner point. */
#define GQM_ARITH_SEPARATE 0
#define GQM_ARITH_CONTRACTED 1
int gqm_arithmetic(void);

#ifdef __cplusplus
}
#endif
#endif
