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
    double  iterate_ms;        /* all sweeps                               */
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

/* Frees a buffer returned by this library. */
void dressx_free(void *p);

#ifdef __cplusplus
}
#endif

#endif /* DRESS_B200_EXT_H */
