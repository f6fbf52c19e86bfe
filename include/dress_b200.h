/*
 * dress_b200.h -- C ABI of the B200 DRESS engine (libdress_cuda.so).
 *
 * The library is a drop-in replacement for libdress's CUDA backend.  It
 * exports every symbol of the reference's CUDA header
 * (libdress/include/dress/cuda/dress_cuda.h:38-110) with identical
 * signatures, plus the graph life-cycle calls that the reference's Python
 * ctypes loader binds from the same shared object
 * (python/src/dress/cuda/__init__.py:142-203).
 *
 * The graph container below is ABI-identical to the reference's
 * dress_graph_t (libdress/include/dress/dress.h:43-75): same member order,
 * types and names, so a graph built by the reference's CPU
 * dress_init_graph() can be passed to these entry points unchanged and
 * vice versa.  If the reference header has already been included
 * (it defines DRESS_H) the shared types are taken from it.
 *
 * Error behaviour: the legacy void / pointer-returning entry points never
 * call exit().  On a CUDA or input error they print one line to stderr,
 * leave the caller's outputs untouched (histogram entry points return NULL
 * with *hist_size = 0) and record the status, which dressx_last_error()
 * returns.  The extended API in dress_b200_ext.h returns the status
 * directly.
 */
#ifndef DRESS_B200_H
#define DRESS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#ifndef DRESS_H
/* (value, count) pair of a Delta/Nabla histogram
 * (reference: libdress/include/dress/dress.h:12-15). */
typedef struct __dress_hist_pair_t {
    double  value;
    int64_t count;
} dress_hist_pair_t;

/* Neighbourhood variant (reference: libdress/include/dress/dress.h:24-29). */
typedef enum __dress_variant_t {
    DRESS_VARIANT_UNDIRECTED = 0,   /* N[u] = N(u), weight 2w            */
    DRESS_VARIANT_DIRECTED   = 1,   /* N[u] = in(u) U out(u)             */
    DRESS_VARIANT_FORWARD    = 2,   /* N[u] = out(u)                     */
    DRESS_VARIANT_BACKWARD   = 3    /* N[u] = in(u)                      */
} dress_variant_t;

/* Graph + fit state (reference: libdress/include/dress/dress.h:43-75).
 * S = adj_offset[N] adjacency slots, T = intercept_offset[E]. */
typedef struct __dress_graph_t {
    dress_variant_t variant;
    int      N;
    int      E;
    int     *U;                 /* [E] edge sources (owned)                   */
    int     *V;                 /* [E] edge targets (owned)                   */
    int     *adj_offset;        /* [N+1] CSR row offsets                      */
    int     *adj_target;        /* [S] neighbour ids, ascending per row       */
    int     *adj_edge_idx;      /* [S] edge id of each slot                   */
    int      max_degree;
    double  *W;                 /* [E] raw weights or NULL                    */
    double  *edge_weight;       /* [E] variant weight w-bar                   */
    double  *edge_dress;        /* [E] current edge values                    */
    double  *edge_dress_next;   /* [E] second buffer                          */
    double  *NW;                /* [N] vertex weights (never NULL after init) */
    double  *vertex_dress;      /* [N] vertex norms of the last sweep         */
    int      precompute_intercepts;
    int     *intercept_offset;  /* [E+1]                                      */
    int     *intercept_edge_ux; /* [T] edge id of (u,x) per common neighbour  */
    int     *intercept_edge_vx; /* [T] edge id of (v,x) per common neighbour  */
} dress_graph_t, *p_dress_graph_t;

/* Graph life cycle.  Same contract as the reference's
 * libdress/include/dress/dress.h:80-83 and :93: takes ownership of the
 * malloc'd U, V, W, NW; builds the variant CSR with rows sorted by
 * neighbour id; initialises every edge value to 1.0.  The CSR, edge
 * weights and intercept tables are bit-identical to the reference's
 * (libdress/src/dress.c:103-427). */
p_dress_graph_t dress_init_graph(int N, int E, int *U, int *V,
                                 double *W, double *NW,
                                 dress_variant_t variant,
                                 int precompute_intercepts);
void dress_free_graph(p_dress_graph_t g);

/* In a CUDA build dress_fit is the GPU fit, as the reference's
 * include-redirect header makes it (libdress/include/dress/cuda/dress.h:27-31);
 * the Python loader binds the name (python/src/dress/cuda/__init__.py:152). */
void dress_fit(p_dress_graph_t g, int max_iterations, double epsilon,
               int *iterations, double *delta);
#endif /* DRESS_H */

/* ---- Entry points of the reference CUDA backend ------------------------ */

/* GPU fixed-point fit of one graph.  Replaces
 * libdress/include/dress/cuda/dress_cuda.h:38-39 (implementation
 * libdress/src/cuda/dress_cuda.cu:445-707).  Same semantics as the CPU
 * dress_fit (libdress/src/dress.c:546-608): continues from g->edge_dress,
 * stops when max|delta| < epsilon, *iterations = 0-based index of the
 * converging sweep (or max_iterations), *delta = last sweep's max change;
 * g->edge_dress and g->vertex_dress are overwritten.  Every sum is the
 * sorted Kahan-Babuska-Neumaier sum of the reference, so results are
 * bit-identical to the CPU fit. */
void dress_fit_cuda(p_dress_graph_t g, int max_iterations, double epsilon,
                    int *iterations, double *delta);

/* Delta^k histogram.  Replaces libdress/include/dress/cuda/dress_cuda.h:47-52
 * (reference driver libdress/src/delta_dress_impl.c:171-318).  All C(N,k)
 * vertex-deleted subgraphs are fitted in one persistent batched launch. */
dress_hist_pair_t *dress_delta_fit_cuda(p_dress_graph_t g, int k, int iterations,
                                        double epsilon,
                                        int n_samples, unsigned int seed,
                                        int *hist_size,
                                        int keep_multisets, double **multisets,
                                        int64_t *num_subgraphs);

/* Replaces libdress/include/dress/cuda/dress_cuda.h:60-66. */
dress_hist_pair_t *dress_delta_fit_cuda_strided(p_dress_graph_t g, int k,
                                                int iterations, double epsilon,
                                                int n_samples, unsigned int seed,
                                                int *hist_size,
                                                int keep_multisets, double **multisets,
                                                int64_t *num_subgraphs,
                                                int offset, int stride);

/* Flat [value_bits, count, ...] form; *hist_size = 2 * distinct values.
 * Replaces libdress/include/dress/cuda/dress_cuda.h:72-78 and the
 * non-strided libdress/src/cuda/delta_dress_cuda.c:24-36. */
int64_t *dress_delta_fit_cuda_strided_flat(p_dress_graph_t g, int k,
                                           int iterations, double epsilon,
                                           int n_samples, unsigned int seed,
                                           int *hist_size,
                                           int keep_multisets, double **multisets,
                                           int64_t *num_subgraphs,
                                           int offset, int stride);
int64_t *dress_delta_fit_cuda_flat(p_dress_graph_t g, int k, int iterations,
                                   double epsilon,
                                   int n_samples, unsigned int seed,
                                   int *hist_size,
                                   int keep_multisets, double **multisets,
                                   int64_t *num_subgraphs);

/* Nabla^k histogram.  Replaces libdress/include/dress/cuda/dress_cuda.h:82-110
 * (reference driver libdress/src/nabla_dress_impl.c:142-311): P(N,k) ordered
 * tuples marked with vertex weights sqrt(prime_i). */
dress_hist_pair_t *dress_nabla_fit_cuda(p_dress_graph_t g, int k, int iterations,
                                        double epsilon,
                                        int n_samples, unsigned int seed,
                                        int *hist_size,
                                        int keep_multisets, double **multisets,
                                        int64_t *num_tuples);
dress_hist_pair_t *dress_nabla_fit_cuda_strided(p_dress_graph_t g, int k,
                                                int iterations, double epsilon,
                                                int n_samples, unsigned int seed,
                                                int *hist_size,
                                                int keep_multisets, double **multisets,
                                                int64_t *num_tuples,
                                                int offset, int stride);
int64_t *dress_nabla_fit_cuda_flat(p_dress_graph_t g, int k, int iterations,
                                   double epsilon,
                                   int n_samples, unsigned int seed,
                                   int *hist_size,
                                   int keep_multisets, double **multisets,
                                   int64_t *num_tuples);
int64_t *dress_nabla_fit_cuda_strided_flat(p_dress_graph_t g, int k,
                                           int iterations, double epsilon,
                                           int n_samples, unsigned int seed,
                                           int *hist_size,
                                           int keep_multisets, double **multisets,
                                           int64_t *num_tuples,
                                           int offset, int stride);

#ifdef __cplusplus
}
#endif

#endif /* DRESS_B200_H */
