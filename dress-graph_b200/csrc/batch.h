// batch.h -- persistent batched fit of many small subgraphs (batch.cu).
#pragma once
#include <stdint.h>

#include <vector>

#include "engine.h"

namespace dress {

enum { ITEM_DELTA = 0, ITEM_NABLA = 1, ITEM_PLAIN = 2 };

// Byte offsets of the packed arrays of one parent graph.  Every section
// starts on a 16-byte boundary so the whole parent can be staged into shared
// memory with 16-byte vector copies.
struct ParentLayout {
    long long U, V, w, row_off, row_eid, ioff, pairs, nw, dinit, bytes;
};

__host__ __device__ inline long long pl_align(long long b) { return (b + 15) & ~15LL; }

__host__ __device__ inline ParentLayout parent_layout(int N, int E, int S, int T, int has_nw, int has_dinit)
{
    ParentLayout L;
    long long o = 0;
    L.U = o;       o = pl_align(o + 4LL * E);
    L.V = o;       o = pl_align(o + 4LL * E);
    L.w = o;       o = pl_align(o + 8LL * E);
    L.row_off = o; o = pl_align(o + 4LL * (N + 1));
    L.row_eid = o; o = pl_align(o + 4LL * S);
    L.ioff = o;    o = pl_align(o + 4LL * (E + 1));
    L.pairs = o;   o = pl_align(o + 8LL * T);
    L.nw = o;      o = pl_align(o + (has_nw ? 8LL * N : 0));
    L.dinit = o;   o = pl_align(o + (has_dinit ? 8LL * E : 0));
    L.bytes = o;
    return L;
}

// Per-request statistics record written by the kernel.
enum { ST_CURSOR = 0, ST_SWEEPS, ST_EDGE_ITERS, ST_FITS, ST_ITERATIONS, ST_DELTA, ST_WORDS };

// One parent graph of a launch and the subgraphs to fit on it.  Every
// pointer addresses device memory owned by the request, so requests of one
// launch may live in unrelated allocations.
struct ParentDesc {
    int N, E, S, T;
    int kind;            // ITEM_*
    int k;
    int fwd;             // FORWARD/BACKWARD self term
    int max_iter;
    double eps;
    int has_nw, has_dinit;
    const unsigned char *data;   // packed arrays (parent_layout)
    double *values;      // DELTA/NABLA: live values in completion order;
                         // PLAIN: E final edge values, then N vertex norms
    unsigned long long *stats;   // ST_WORDS counters
    double *multisets;   // C(N,k) x E row-major matrix, or null
    const long long *ranks;      // sampled ranks (item i -> ranks[i]), or null ...
    long long offset, stride;    // ... else rank of item i = offset + i*stride
    int force_exact;             // every sum by the exact sorted path (tests of that path)
};

struct Chunk {
    int parent;
    int count;
    long long first;     // first item index within the parent
};

struct BatchLaunch {
    const ParentDesc *parents;
    const Chunk *chunks;
    int nchunks;
    int *chunk_counter;
    int gsize, groups;               // threads per subgraph, subgraphs per CTA
    int stage;                       // parents copied into shared memory (CTA mode)
    int per_group;                   // every group takes its own chunks (no staging)
    int min_ctas;                    // CTAs per SM the schedule is built for (1 or 2)
    int maxE, maxN, maxk;            // per-group state sizes
    long long parent_bytes;          // staging area size
    int M;                           // most terms of any item (a row or an edge's pairs, plus one)
};

Status launch_batch(const BatchLaunch &L, int sms, cudaStream_t st);
// One whole-graph fit (the ITEM_PLAIN descriptor at d_parent) by one cluster
// of 2^lnc CTAs whose shared memory holds the state (cluster_fit_smem_bytes
// per CTA).  DRESSX_EUNSUPPORTED when such a cluster cannot be placed.
Status launch_cluster_fit(const ParentDesc *d_parent, int E, int N, int lnc, int sms, cudaStream_t st);
size_t cluster_fit_smem_bytes(int E, int N, int lnc);
size_t batch_smem_bytes(const BatchLaunch &L);
// Shared memory of one group's state (edge values twice, vertex norms,
// reduction slots, the k mask vertices); a graph is batchable only when one
// group fits, with room left for the kernel's static shared memory.
long long batch_group_bytes(int maxE, int maxN, int maxk, int gsize);
constexpr long long BATCH_GROUP_BYTES_MAX = 226 * 1024;

// ---- host planning helpers (delta_nabla.cpp) ------------------------------------
long long binom_h(int n, int k);
long long perm_h(int n, int k);
// Common-neighbour pairs of every edge by the reference's merge walk
// (libdress/src/dress.c:307-363): pairs[2t], pairs[2t+1] are the (u,x) and
// (v,x) edge ids of pair t, ioff[e]..ioff[e+1] the pairs of edge e.  Also the
// largest row and whether any row repeats a neighbour.
void merge_walk_pairs(p_dress_graph_t g, std::vector<int> &ioff, std::vector<int> &pairs, int &maxdeg, bool &dup);

}  // namespace dress
