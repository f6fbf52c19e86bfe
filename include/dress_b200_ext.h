/*
 * dress_b200_ext.h -- extended C ABI of the B200 DRESS engine.
 *
 * The reference has no counterpart for these calls: its CUDA backend
 * prints and exit()s on error (libdress/src/cuda/dress_cuda.cu:41-49) and
 * fits one graph per call.  The calls below return an int status instead
 * and batch many Delta/Nabla requests into one persistent launch; the
 * legacy entry points of dress_b200.h are thin wrappers over them.
 */
#ifndef DRESS_B200_EXT_H
#define DRESS_B200_EXT_H

#include <stddef.h>
#include <stdint.h>
#include "dress_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes returned by every dressx_* call. */
enum {
    DRESSX_OK           = 0,
    DRESSX_EINVAL       = 1,   /* malformed graph or argument              */
    DRESSX_ENOMEM       = 2,   /* device or host allocation refused        */
    DRESSX_ECUDA        = 3,   /* CUDA runtime error                       */
    DRESSX_ETIMEOUT     = 4,   /* a bounded device wait gave up            */
    DRESSX_EUNSUPPORTED = 5,   /* request outside the engine's limits      */
    DRESSX_EBUDGET      = 6,   /* request larger than the memory budget    */
    DRESSX_ECANCELLED   = 7,   /* request cancelled before it ran          */
    DRESSX_EBUSY        = 8    /* server queue full                        */
};

/* Engine configuration (process-wide).  Zero fields take defaults. */
typedef struct dressx_config_t {
    int     device;               /* CUDA device ordinal; -1 = current        */
    size_t  memory_budget_bytes;  /* device memory the engine may hold        */
    int     fit_chunk;            /* sweeps launched per convergence check    */
    int     group_threads;        /* threads per subgraph in the batch kernel;
                                     0 = pick from the tuned table            */
    int     exact_sums;           /* 1 = every sum takes the sorted path (the
                                     fallback of the certified sums; slower,
                                     same bits); for testing that path        */
    int     one_launch_max_edges; /* graphs up to this many edges are fitted
                                     in one launch; 0 = built-in limit,
                                     -1 = never                               */
    int     reserved[6];
} dressx_config_t;

/* Replace the engine configuration; call before the first fit. */
int dressx_configure(const dressx_config_t *cfg);

/* Status of the last failing call on any thread, and its message. */
int dressx_last_error(char *msg, int msg_len);

/* Status-returning form of dress_fit_cuda. */
int dressx_fit(p_dress_graph_t g, int max_iterations, double epsilon,
               int *iterations, double *delta);

/* Per-sweep statistics of the last dressx_fit on this process. */
typedef struct dressx_fit_stats_t {
    int64_t common_terms;      /* sum over edges of |N[u] ^ N[v]|          */
    int     sweeps;            /* sweeps executed                          */
    double  setup_ms;          /* upload + intercepts + binning            */
    double  iterate_ms;        /* all sweeps, device time (CUDA events)    */
    /* items and stored terms per size bin (0, <=2, <=4, <=8, <=16, <=512,
     * <=4096, more terms), vertices (row slots) and edges (common pairs) */
    int64_t vertex_bin_items[8], vertex_bin_terms[8];
    int64_t edge_bin_items[8], edge_bin_terms[8];
    /* host time of the phases: upload, validation, common-neighbour tables
     * and bins, renumbering and sweep set-up, download of the results */
    double  phase_ms[5];
} dressx_fit_stats_t;
int dressx_last_fit_stats(dressx_fit_stats_t *out);

/* One Delta^k or Nabla^k histogram request. */
enum { DRESSX_DELTA = 0, DRESSX_NABLA = 1 };

typedef struct dressx_hist_request_t {
    /* inputs */
    p_dress_graph_t graph;       /* topology (and raw W, variant) to use     */
    int      kind;               /* DRESSX_DELTA or DRESSX_NABLA             */
    int      k;
    int      max_iterations;
    double   epsilon;
    int      n_samples;          /* 0 = all subsets / tuples of the stride   */
    unsigned int seed;
    int      offset, stride;     /* process index s with s % stride == offset */
    int      want_histogram;     /* 0 = skip the histogram                   */
    int      keep_multisets;     /* 1 = fill a [num_subgraphs x E] matrix    */
    /* outputs (malloc'd; the caller frees them with free()) */
    int64_t *hist_flat;          /* [value_bits, count, ...] ascending       */
    int      hist_len;           /* 2 * distinct values                      */
    double  *multisets;          /* row s, edge e at [s*E + e]; NaN = absent */
    int64_t  num_subgraphs;      /* C(N,k) or P(N,k)                         */
    int64_t  fits;               /* subgraphs fitted by this request         */
    int      status;
} dressx_hist_request_t;

/* Run n requests.  Small graphs from all requests share one persistent
 * launch; each request's histogram is exact and independent of the others
 * in the batch.  Returns the first failing status (each request also
 * carries its own). */
int dressx_hist_batch(dressx_hist_request_t *reqs, int n);

/* Same as dressx_hist_batch, but every subgraph goes through the
 * per-subgraph path: host-built subgraph CSR + one single-graph GPU fit per
 * subgraph, the structure of the reference driver
 * (libdress/src/delta_dress_impl.c:268-309).  Kept as the baseline the
 * batched engine is measured against. */
int dressx_hist_batch_per_fit(dressx_hist_request_t *reqs, int n);

/* A prepared batch: the requests' graphs packed and resident in device
 * memory, so the fits and histograms can be re-run without host traffic.
 * Every request must be batchable (k >= 1, rows of at most 31 neighbours);
 * dressx_batch_create returns DRESSX_EUNSUPPORTED otherwise.  The requests
 * must stay alive until dressx_batch_destroy. */
typedef struct dressx_batch dressx_batch_t;
int  dressx_batch_create(dressx_hist_request_t *reqs, int n, dressx_batch_t **out);
/* All fits and histograms on the device; results stay in device memory. */
int  dressx_batch_run(dressx_batch_t *b);
/* Autotuner: runs the batch kernel on this batch's subgraphs (a spread
 * sample beyond 200K) with 32, 64, 128 and 256 threads per subgraph and one
 * 512-thread CTA per SM, then 32, 64 and 128 threads with two CTAs sharing
 * each SM -- each schedule where one subgraph's state fits shared memory --
 * timing the median of three runs after an untimed one.  It keeps the first
 * schedule, in that order, within 3 % of the fastest (so schedules closer
 * than the run-to-run noise resolve the same way every time) for the
 * batch's size class (batches of that class planned later in the process
 * start from it) and re-plans this batch with it.  *group_threads and
 * *ctas_per_sm (nullable) get the winner; rates[8] (nullable) the
 * subgraph-fits per ms of the candidates in that order (0 = did not fit). */
int  dressx_batch_autotune(dressx_batch_t *b, int *group_threads, int *ctas_per_sm, float *rates);
/* Captures the fit stage (counter resets and the batch kernel) into a CUDA
 * graph; later dressx_batch_run calls replay it with one launch. */
int  dressx_batch_capture(dressx_batch_t *b);
/* Copies the last run's histograms (and multisets) into the requests. */
int  dressx_batch_fetch(dressx_batch_t *b);
/* Totals of the last run: subgraphs fitted, sweeps, live-edge updates. */
int  dressx_batch_stats(dressx_batch_t *b, int64_t *fits, int64_t *sweeps, int64_t *edge_updates);
/* Device time of the last run, from CUDA events on the engine stream:
 * the batched fit kernel, and the histogram kernels after it. */
int  dressx_batch_timing(dressx_batch_t *b, double *fit_ms, double *hist_ms);
void dressx_batch_destroy(dressx_batch_t *b);

/* The engine's CUDA stream (cudaStream_t) -- every kernel of this library
 * is launched on it, so callers can time them with events on this stream. */
int dressx_stream(void **stream);

/* Counters since the last reset: bytes copied host->device and
 * device->host by this library, and kernels it launched. */
int dressx_counters(int64_t *h2d_bytes, int64_t *d2h_bytes, int64_t *launches, int reset);

/* ---- Histogram without allocation -------------------------------------
 * No counterpart in the reference.  Exact (value, count) histogram of n
 * doubles that already sit in device memory, for callers that cannot
 * allocate device memory when they need it: code running while a CUDA graph
 * is captured, frameworks whose caching allocator owns the device memory,
 * and loops that must not allocate after start-up.  The call allocates
 * nothing: its scratch is one fixed array of about 16.5 MiB compiled into the
 * library, which every GPU that loads the library holds until the process
 * exits.
 *   values   device pointer, n doubles (n <= DRESSX_NOALLOC_MAX_VALUES;
 *            larger n returns DRESSX_EUNSUPPORTED and enqueues nothing)
 *   pairs    device pointer, room for 2*n int64: [value bits, count, ...]
 *            ascending by value, one entry per bit pattern (+0 and -0
 *            apart, every NaN apart) as in dressx_hist_batch
 *   num_runs device pointer, one int64: the number of (value, count) pairs
 *   stream   cudaStream_t the work is enqueued on (NULL = legacy stream)
 * Nothing is synchronised: results are valid once the stream has run the
 * enqueued work.  A call made outside stream capture looks up the array's
 * device address in the current context (so a device reset or a switch of
 * context is followed); a call on a stream under capture reuses the address
 * of the device's last call outside capture, so make the first call on a
 * device before any stream capture starts.  Every
 * call uses the same array, so calls whose work overlaps on the GPU (other
 * streams, other host threads) race and must be serialised by the caller. */
#define DRESSX_NOALLOC_MAX_VALUES (1 << 20)
int dressx_histogram_noalloc(const double *values, int64_t n, int64_t *pairs, int64_t *num_runs,
                             void *stream);

/* dress_init_graph built on the GPU: same arguments, ownership rules and
 * result -- array for array bit-identical to the host build (and to the
 * reference, libdress/src/dress.c:378-427) -- with the row sorting, the
 * variant weights and the intercept tables computed on the device.  NULL on
 * an invalid graph or a device error (dressx_last_error); the caller then
 * keeps U, V, W and NW.  Free the result with dress_free_graph. */
p_dress_graph_t dressx_init_graph(int N, int E, int *U, int *V, double *W, double *NW,
                                  dress_variant_t variant, int precompute_intercepts);

/* Batched virtual-edge queries on a fitted graph: out[i] is what the
 * reference's dress_get(g, u[i], v[i], max_iterations, epsilon, w) returns
 * (libdress/include/dress/dress.h:105, libdress/src/dress.c:651-739) -- the
 * stored value of an existing edge, else the pair's own fixed point with
 * every other value frozen -- with w = edge_weights[i], or edge_weight when
 * edge_weights is NULL.  u, v, edge_weights and out are host arrays of n
 * entries; the graph's current edge and vertex values are used.  A vertex
 * out of range fails the call with DRESSX_EINVAL. */
int dressx_get_batch(p_dress_graph_t g, const int *u, const int *v, int64_t n, int max_iterations,
                     double epsilon, const double *edge_weights, double edge_weight, double *out);

/* Merge of histograms computed on disjoint shards of one request (e.g. the
 * strided slices offset = rank, stride = ranks of several GPUs or
 * processes): n flat [value_bits, count, ...] lists, each ascending by value,
 * into one list of the same form (malloc'd; *out_len entries).  Counts of
 * equal bit patterns add up (a NaN stays an entry of its own).  Replaces the gather-and-reinsert step of the
 * reference's MPI layer (libdress/src/mpi/dress_mpi.c:90-118). */
int dressx_hist_merge(const int64_t *const *flats, const int64_t *lens, int n, int64_t **out,
                      int64_t *out_len);

/* ---- Request server ----------------------------------------------------
 * No counterpart in the reference: its CUDA backend fits one graph per call
 * on the legacy stream.  A server takes fit and Delta/Nabla requests from
 * any number of host threads as they arrive and serves them concurrently:
 *   - admission: a request reserves an estimate of its device memory from
 *     the server's budget; requests wait in arrival order until it fits
 *     (one larger than the whole budget fails with DRESSX_EBUDGET);
 *   - residency: admitted requests keep their packed graph and edge state in
 *     the server's own memory pool (an arena that keeps its memory between
 *     requests) until they complete;
 *   - continuous batching: small requests (every row of at most 31
 *     neighbours, state within shared memory; whole-graph fits up to 2048
 *     edges) are cut into slices and packed
 *     into short persistent batch launches, a few in flight at once; a
 *     request that arrives while launches run joins the next launch, every
 *     waiting request gets a share of each launch, and a request completes as
 *     soon as its last slice has run;
 *   - lanes: larger requests run on their own streams (the single-graph fit,
 *     or the per-subgraph Delta/Nabla path), beside the batch launches;
 *   - latency: each request records its queueing and end-to-end time; the
 *     statistics give p50/p99 per class.
 * Results are bit-identical to the single-request calls (dressx_fit,
 * dressx_hist_batch), whatever else is in service. */
typedef struct dressx_server dressx_server_t;

typedef struct dressx_server_config_t {
    int     device;               /* CUDA device ordinal; -1 = current        */
    size_t  memory_budget_bytes;  /* admission budget; 0 = 120 GiB, at most
                                     90% of the device memory free at create */
    int     lanes;                /* concurrent large requests; 0 = 4          */
    int     launch_slots;         /* batch launches in flight; 0 = 3           */
    int64_t launch_work;          /* edge-subgraph units per batch launch
                                     (sum of edges over its fits); 0 = 2^21   */
    int     finishers;            /* threads building results; 0 = 2           */
    int     max_queued;           /* requests waiting for admission; 0 = 65536 */
    int     reserved[8];
} dressx_server_config_t;

/* Request kinds: DRESSX_DELTA, DRESSX_NABLA (above) and a plain fit. */
enum { DRESSX_FIT = 2 };

/* Where a request was served. */
enum { DRESSX_PATH_NONE = 0, DRESSX_PATH_BATCH = 1, DRESSX_PATH_LANE = 2 };

/* Statistics classes: kind x path. */
enum { DRESSX_CLASS_FIT_BATCH = 0, DRESSX_CLASS_FIT_LANE = 1,
       DRESSX_CLASS_HIST_BATCH = 2, DRESSX_CLASS_HIST_LANE = 3, DRESSX_CLASSES = 4 };

typedef struct dressx_server_request_t {
    /* inputs; the graph must stay alive and unchanged until `done` */
    p_dress_graph_t graph;
    int      kind;               /* DRESSX_FIT, DRESSX_DELTA, DRESSX_NABLA   */
    int      k;                  /* Delta/Nabla order                        */
    int      max_iterations;
    double   epsilon;
    /* outputs.  DRESSX_FIT updates graph->edge_dress and vertex_dress in
     * place, as dress_fit does, and sets iterations / delta (delta is left
     * as it was when max_iterations <= 0).  Delta/Nabla return the exact
     * histogram, malloc'd (free with free() or dressx_free). */
    int      iterations;
    double   delta;
    int64_t *hist_flat;          /* [value_bits, count, ...] ascending       */
    int      hist_len;           /* 2 * distinct values                      */
    int64_t  num_subgraphs;      /* C(N,k) or P(N,k)                         */
    int64_t  fits;               /* fits run for this request                */
    int64_t  edge_sweeps;        /* sum over fits of live edges x sweeps     */
    int      path;               /* DRESSX_PATH_*                            */
    int      status;             /* DRESSX_* of this request                 */
    double   queue_ms;           /* submission -> admission                  */
    double   latency_ms;         /* submission -> completion                 */
    int64_t  reserved_bytes;     /* device memory reserved at admission      */
    volatile int done;           /* 1 once every output above is final       */
} dressx_server_request_t;

typedef struct dressx_server_class_stats_t {
    int64_t completed, failed;
    double  p50_ms, p99_ms, mean_ms, max_ms;     /* end-to-end latency       */
    double  queue_p50_ms, queue_p99_ms;          /* waiting for admission    */
} dressx_server_class_stats_t;

typedef struct dressx_server_stats_t {
    double   elapsed_s;           /* since create or the last reset          */
    int64_t  submitted, completed, failed, cancelled, rejected;
    int64_t  fits;                /* subgraph and graph fits completed       */
    int64_t  edge_sweeps;         /* live edges x sweeps over those fits     */
    int64_t  batch_launches;
    int64_t  budget_bytes, reserved_bytes, peak_reserved_bytes;
    int64_t  pool_bytes;          /* device memory the arena pool holds      */
    int      max_in_service;      /* most requests admitted at once          */
    double   device_busy_ms;      /* union of the device intervals of batch
                                     launches and lane requests              */
    double   device_work_ms;      /* their sum (> busy when work overlapped) */
    dressx_server_class_stats_t cls[DRESSX_CLASSES];
} dressx_server_stats_t;

int  dressx_server_create(const dressx_server_config_t *cfg, dressx_server_t **out);
/* Queue a request (the struct must stay alive until done).  Returns
 * DRESSX_OK once queued; a request refused at once (bad arguments, larger
 * than the budget, queue full) returns its status and is marked done. */
int  dressx_server_submit(dressx_server_t *s, dressx_server_request_t *req);
/* Wait until req is done: its status, or DRESSX_ETIMEOUT after timeout_ms
 * (negative = no limit). */
int  dressx_server_wait(dressx_server_t *s, dressx_server_request_t *req, int timeout_ms);
/* Cancel a request that has not started device work (DRESSX_OK; it ends
 * with DRESSX_ECANCELLED), or a Delta/Nabla batch request between slices;
 * DRESSX_EBUSY when it is too late. */
int  dressx_server_cancel(dressx_server_t *s, dressx_server_request_t *req);
/* Wait until no request is queued or in service. */
int  dressx_server_drain(dressx_server_t *s, int timeout_ms);
int  dressx_server_stats(dressx_server_t *s, dressx_server_stats_t *out, int reset);
/* Cancels queued requests, finishes admitted ones, frees the arena. */
int  dressx_server_destroy(dressx_server_t *s);

/* Host-only planning of a request (no device needed): the device memory it
 * would reserve and the path it would take. */
int  dressx_server_estimate(p_dress_graph_t g, int kind, int k, int64_t *bytes, int *path);

/* Frees a buffer returned by this library. */
void dressx_free(void *p);

#ifdef __cplusplus
}
#endif

#endif /* DRESS_B200_EXT_H */
