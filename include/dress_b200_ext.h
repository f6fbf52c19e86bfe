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
    int     reserved[8];
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
 *            ascending by value, ==-equal values merged as in
 *            dressx_hist_batch
 *   num_runs device pointer, one int64: the number of (value, count) pairs
 *   stream   cudaStream_t the work is enqueued on (NULL = legacy stream)
 * Nothing is synchronised: results are valid once the stream has run the
 * enqueued work.  The first call on a device looks up the array's device
 * address; make that first call before any stream capture starts.  Every
 * call uses the same array, so calls whose work overlaps on the GPU (other
 * streams, other host threads) race and must be serialised by the caller. */
#define DRESSX_NOALLOC_MAX_VALUES (1 << 20)
int dressx_histogram_noalloc(const double *values, int64_t n, int64_t *pairs, int64_t *num_runs,
                             void *stream);

/* Frees a buffer returned by this library. */
void dressx_free(void *p);

#ifdef __cplusplus
}
#endif

#endif /* DRESS_B200_EXT_H */
