// batch.h -- persistent batched fit of many small subgraphs (batch.cu).
#pragma once
#include <stdint.h>

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

// One parent graph of a launch and the subgraphs to fit on it.
struct ParentDesc {
    int N, E, S, T;
    int kind;            // ITEM_*
    int k;
    int fwd;             // FORWARD/BACKWARD self term
    int max_iter;
    double eps;
    int has_nw, has_dinit;
    int req;             // request slot (value cursor, statistics)
    int pad;
    long long data_off;  // byte offset of the packed arrays in the parent arena
    long long offset, stride;   // rank of item i = offset + i*stride ...
    long long ranks_off; // ... or ranks[ranks_off + i] when >= 0 (sampling)
    long long val_base;  // first slot of this request's value segment
    long long ms_base;   // multiset matrix of this request, -1 = none
    long long E_ms;      // row length of the multiset matrix
};

struct Chunk {
    int parent;
    int count;
    long long first;     // first item index within the parent
};

struct BatchLaunch {
    const ParentDesc *parents;
    const unsigned char *pdata;
    const Chunk *chunks;
    int nchunks;
    int *chunk_counter;
    const long long *ranks;
    double *values;
    unsigned long long *cursors;     // per request: values written
    unsigned long long *sweeps;      // per request: sum of sweeps over fits
    unsigned long long *edge_iters;  // per request: sum of live edges x sweeps
    unsigned long long *fits;        // per request: subgraphs fitted
    double *multisets;
    int gsize, groups;               // threads per subgraph, subgraphs per CTA
    int stage;                       // parents copied into shared memory
    int maxE, maxN, maxk;            // per-group state sizes
    long long parent_bytes;          // staging area size
    int M;                           // register network size (max terms)
};

Status launch_batch(const BatchLaunch &L, int sms, cudaStream_t st);
size_t batch_smem_bytes(const BatchLaunch &L);

}  // namespace dress
