// fit_small.cu -- the single-graph fit of a small or mid-size graph in one launch.
//
// Reference: libdress/src/dress.c:546-608 (the iteration driver) with the
// vertex and edge phases of :556-591.  A graph whose whole fit state (edge
// values twice, vertex norms) fits one SM's shared memory, with rows of at
// most 256 neighbours, is fitted by one 512-thread CTA of the batch kernel as
// a single whole-graph item: every sweep, the convergence test and the final
// values in one launch, without per-sweep kernels or host round trips.  The
// arithmetic is the batch kernel's, bit-identical to the reference's
// (certified sums with the sorted Kahan-Babuska-Neumaier sum as their
// fallback, separately rounded products).  The graph is
// staged in shared memory as well.  Graphs of up to CLUSTER_MAX_EDGES edges
// that do not fit one CTA run on a thread-block cluster instead, the state
// spread over its CTAs' distributed shared memory (batch.cu,
// k_fit_cluster).  Larger graphs, and graphs that carry their own intercept
// tables, take the multi-kernel fit in fit_graph.cu.
#include <algorithm>
#include <climits>
#include <chrono>
#include <cstring>
#include <vector>

#include "batch.h"
#include "engine.h"

namespace dress {

namespace {
constexpr int SMALL_GSIZE = 512;       // threads of the one group
// Above about 3000 edges one SM takes longer than the multi-kernel fit over
// the whole device (measured on G(n, m): 0.21-0.33 ms against 0.95 ms up to
// 1500 edges, even at 3000, behind beyond).
constexpr int SMALL_MAX_EDGES = 2048;
// Beyond that, up to this many edges, one cluster of 8 (or 16) CTAs holds
// the state in its distributed shared memory and runs the fit in one
// launch.  Measured per dress_fit_cuda call on G(n, m), one launch against
// the multi-kernel fit: 0.39 / 1.10 ms at 3000 edges, 0.61 / 1.16 ms at
// 8000, 0.70 / 1.19 ms at 10000, 0.87 / 1.23 ms at 15000, 1.10 / 1.27 ms at
// 20000, 2.49 / 1.43 ms at 40000 (a cluster's per-thread load chains are
// latency-bound, the multi-kernel fit pays about 1 ms of fixed cost).
constexpr int CLUSTER_MAX_EDGES = 24576;
// Rows up to this many neighbours: one thread sums an item's terms, so a
// longer row would make one thread's serial loop the whole sweep; the
// multi-kernel fit gives such rows a warp or a block.
constexpr int SMALL_MAX_DEG = 256;

// The checks of fit_graph's device validation, on the host: rows in order
// and in range, edge ids and endpoints in range.
bool small_graph_ok(p_dress_graph_t g, int &maxdeg)
{
    const int N = g->N, E = g->E;
    maxdeg = 0;
    for (int u = 0; u < N; ++u) {
        const int b = g->adj_offset[u], e = g->adj_offset[u + 1];
        if (e < b) return false;
        maxdeg = std::max(maxdeg, e - b);
        for (int s = b; s < e; ++s) {
            const int x = g->adj_target[s], ei = g->adj_edge_idx[s];
            if (x < 0 || x >= N || ei < 0 || ei >= E) return false;
            if (s > b && x < g->adj_target[s - 1]) return false;
        }
    }
    for (int e = 0; e < E; ++e)
        if (g->U[e] < 0 || g->U[e] >= N || g->V[e] < 0 || g->V[e] >= N) return false;
    return true;
}

// Common-neighbour pairs of a graph for the cluster fit, on the device: one
// block.  Each thread runs the reference's merge walk (dress.c:500-529) over
// the rows of its edges -- counts first, then a block scan of the counts
// into the offsets, then the same walk writes the pairs, in the walk's
// order.  Rows and offsets are staged in shared memory when they fit.
constexpr int PAIR_THR = 1024;

__global__ void __launch_bounds__(PAIR_THR) k_small_pairs(int N, int E, const int *off_g, const int *tgt_g,
                                                          const int *eidx, const int *U, const int *V, int *ioff,
                                                          int2 *pairs, int staged)
{
    extern __shared__ __align__(16) int sm[];
    __shared__ int part[PAIR_THR / 32];
    const int *off = off_g, *tgt = tgt_g;
    const long long S = off_g[N];
    if (staged) {
        int *so = sm, *st = sm + N + 1;
        for (int i = threadIdx.x; i <= N; i += blockDim.x) so[i] = off_g[i];
        for (long long i = threadIdx.x; i < S; i += blockDim.x) st[i] = tgt_g[i];
        __syncthreads();
        off = so;
        tgt = st;
    }
    // this thread's edges: a contiguous chunk, so the scan is a chunk sum
    const int per = (E + (int)blockDim.x - 1) / (int)blockDim.x;
    const int e0 = min(E, (int)threadIdx.x * per), e1 = min(E, e0 + per);
    int mine = 0;
    for (int e = e0; e < e1; ++e) {
        int iu = off[U[e]], iu_end = off[U[e] + 1];
        int iv = off[V[e]], iv_end = off[V[e] + 1];
        int c = 0;
        while (iu < iu_end && iv < iv_end) {
            const int x = tgt[iu], y = tgt[iv];
            c += x == y;
            iu += (x <= y);
            iv += (x >= y);
        }
        ioff[e + 1] = c;          // counts for now
        mine += c;
    }
    // exclusive block scan of the chunk sums
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int incl = mine;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) part[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        int v = lane < (int)(blockDim.x >> 5) ? part[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += y;
        }
        if (lane < (int)(blockDim.x >> 5)) part[lane] = v;
    }
    __syncthreads();
    int base = incl - mine + (wid > 0 ? part[wid - 1] : 0);
    if (threadIdx.x == 0) ioff[0] = 0;
    for (int e = e0; e < e1; ++e) {
        const int c = ioff[e + 1];
        int iu = off[U[e]], iu_end = off[U[e] + 1];
        int iv = off[V[e]], iv_end = off[V[e] + 1];
        int q = base;
        while (iu < iu_end && iv < iv_end) {
            const int x = tgt[iu], y = tgt[iv];
            if (x == y) pairs[q++] = make_int2(eidx[iu], eidx[iv]);
            iu += (x <= y);
            iv += (x >= y);
        }
        base += c;
        ioff[e + 1] = base;
    }
}

}  // namespace

Status fit_small(p_dress_graph_t g, int max_iterations, double epsilon, int *iterations, double *delta,
                 FitStats *stats, const Ctx &ctx, bool &used)
{
    used = false;
    const auto t0 = std::chrono::steady_clock::now();
    const int N = g->N, E = g->E;
    const int max_edges = ctx.cfg->one_launch_max_edges == 0 ? CLUSTER_MAX_EDGES : ctx.cfg->one_launch_max_edges;
    if (E < 1 || E > max_edges || N < 1 || (g->precompute_intercepts && g->intercept_offset))
        return Status::Ok();
    const long long S = g->adj_offset[N];
    if (g->adj_offset[0] != 0 || S < 0) return Status::Ok();      // fit_graph reports it

    // shape: one group of SMALL_GSIZE threads and the staged parent (the state
    // and the graph without its pairs must fit before the pairs are found),
    // else a cluster of 8 CTAs (16 when 8 cannot hold the state)
    int smem_optin = 0;
    DRESS_CUDA_TRY(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx.device));
    const long long smem_cap = smem_optin - 1024;
    bool one_cta = E <= SMALL_MAX_EDGES &&
                   batch_group_bytes(E, N, 1, SMALL_GSIZE) +
                           parent_layout(N, E, (int)S, 0, g->NW != nullptr, 1).bytes <= smem_cap;
    int lnc = -1;
    if (!one_cta) {
        if ((long long)cluster_fit_smem_bytes(E, N, 3) <= smem_cap) lnc = 3;
        else if ((long long)cluster_fit_smem_bytes(E, N, 4) <= smem_cap) lnc = 4;
        else return Status::Ok();
    }
    int maxdeg = 0;
    if (!small_graph_ok(g, maxdeg)) return Status::Ok();       // fit_graph reports it
    if (maxdeg > SMALL_MAX_DEG) return Status::Ok();

    // the common-neighbour pairs: on the host for one CTA (whose staged
    // image must be exact), on the device for a cluster, in an image sized
    // for the bound T <= sum_e min(deg u, deg v)
    std::vector<int> ioff, pairs;
    long long T = 0;
    if (one_cta) {
        bool dup = false;                    // repeated neighbours: the merge walk pairs them as the reference does
        merge_walk_pairs(g, ioff, pairs, maxdeg, dup);
        T = (long long)(pairs.size() / 2);
    } else {
        for (int e = 0; e < E; ++e) {
            const int du = g->adj_offset[g->U[e] + 1] - g->adj_offset[g->U[e]];
            const int dv = g->adj_offset[g->V[e] + 1] - g->adj_offset[g->V[e]];
            T += du < dv ? du : dv;
        }
        if (T > INT_MAX / 2) return Status::Ok();
    }
    const int has_nw = g->NW != nullptr;
    const ParentLayout PL = parent_layout(N, E, (int)S, (int)T, has_nw, 1);

    BatchLaunch L{};
    L.gsize = SMALL_GSIZE;
    L.groups = 1;
    L.per_group = 0;
    L.min_ctas = 1;
    L.maxE = E;
    L.maxN = N;
    L.maxk = 1;
    L.M = maxdeg + 1;
    L.parent_bytes = PL.bytes;
    // On one CTA the graph itself must be staged in shared memory too: read
    // through L2 by a single SM, the sweeps are latency-bound and the
    // multi-kernel fit answers sooner (measured on G(2000, 10000): 3.9 ms
    // against 1.3 ms).
    L.stage = 1;
    if (one_cta && (long long)batch_smem_bytes(L) > smem_cap) {
        one_cta = false;
        if ((long long)cluster_fit_smem_bytes(E, N, 3) <= smem_cap) lnc = 3;
        else if ((long long)cluster_fit_smem_bytes(E, N, 4) <= smem_cap) lnc = 4;
        else return Status::Ok();
    }

    // One device block holds everything: the packed parent image, the row
    // targets (cluster: the device pair walk reads them), the descriptor, the
    // chunk, the counter, the statistics and the results.  The host writes
    // the inputs once, into the context's pinned stage, and one copy each
    // way moves them.
    auto al = [](size_t x) { return (x + 15) & ~(size_t)15; };
    const size_t off_tgt = al((size_t)PL.bytes);
    const size_t off_desc = al(off_tgt + (one_cta ? 0 : (size_t)S * sizeof(int)));
    const size_t off_chunk = al(off_desc + sizeof(ParentDesc));
    const size_t off_ctr = al(off_chunk + sizeof(Chunk));
    const size_t off_stats = al(off_ctr + sizeof(int));
    const size_t off_vals = al(off_stats + ST_WORDS * sizeof(unsigned long long));
    const size_t total = off_vals + ((size_t)E + N) * sizeof(double);
    cudaStream_t st = ctx.st;
    DevBuf<unsigned char> d_blob;
    DRESS_TRY(d_blob.alloc(total, st));
    DRESS_TRY(ctx.stage->reserve(total));
    unsigned char *h = (unsigned char *)ctx.stage->ptr();
    unsigned char *dv = d_blob.get();
    std::memcpy(h + PL.U, g->U, (size_t)E * 4);
    std::memcpy(h + PL.V, g->V, (size_t)E * 4);
    std::memcpy(h + PL.w, g->edge_weight, (size_t)E * 8);
    std::memcpy(h + PL.row_off, g->adj_offset, (size_t)(N + 1) * 4);
    if (S) std::memcpy(h + PL.row_eid, g->adj_edge_idx, (size_t)S * 4);
    if (one_cta) {
        std::memcpy(h + PL.ioff, ioff.data(), (size_t)(E + 1) * 4);
        if (T) std::memcpy(h + PL.pairs, pairs.data(), (size_t)T * 8);
    } else if (S) {
        std::memcpy(h + off_tgt, g->adj_target, (size_t)S * 4);
    }
    if (has_nw) std::memcpy(h + PL.nw, g->NW, (size_t)N * 8);
    std::memcpy(h + PL.dinit, g->edge_dress, (size_t)E * 8);
    ParentDesc P{};
    P.N = N;
    P.E = E;
    P.S = (int)S;
    P.T = (int)T;
    P.kind = ITEM_PLAIN;
    P.k = 0;
    P.fwd = g->variant == DRESS_VARIANT_FORWARD || g->variant == DRESS_VARIANT_BACKWARD;
    P.force_exact = ctx.cfg->exact_sums != 0;
    P.max_iter = max_iterations;
    P.eps = epsilon;
    P.has_nw = has_nw;
    P.has_dinit = 1;
    P.data = dv;
    P.values = (double *)(dv + off_vals);
    P.stats = (unsigned long long *)(dv + off_stats);
    P.offset = 0;
    P.stride = 1;
    const Chunk ch{0, 1, 0};
    std::memcpy(h + off_desc, &P, sizeof P);
    std::memcpy(h + off_chunk, &ch, sizeof ch);
    std::memset(h + off_ctr, 0, off_vals - off_ctr);           // counter and statistics
    DRESS_CUDA_TRY(counted_memcpy(dv, h, off_vals, cudaMemcpyHostToDevice, st));
    if (!one_cta) {
        const size_t pair_smem = (size_t)(N + 1 + S) * sizeof(int);
        const int staged = pair_smem <= (size_t)smem_cap ? 1 : 0;
        static bool attr_set[64] = {};
        if (staged && ctx.device >= 0 && ctx.device < 64 && !attr_set[ctx.device]) {
            DRESS_CUDA_TRY(cudaFuncSetAttribute(k_small_pairs, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_cap));
            attr_set[ctx.device] = true;
        }
        count_launch(), k_small_pairs<<<1, PAIR_THR, staged ? pair_smem : 0, st>>>(
            N, E, (const int *)(dv + PL.row_off), (const int *)(dv + off_tgt), (const int *)(dv + PL.row_eid),
            (const int *)(dv + PL.U), (const int *)(dv + PL.V), (int *)(dv + PL.ioff), (int2 *)(dv + PL.pairs), staged);
        DRESS_CUDA_TRY(cudaGetLastError());
    }
    L.parents = (const ParentDesc *)(dv + off_desc);
    L.chunks = (const Chunk *)(dv + off_chunk);
    L.nchunks = 1;
    L.chunk_counter = (int *)(dv + off_ctr);

    cudaEvent_t e0, e1;
    DRESS_CUDA_TRY(cudaEventCreate(&e0));
    DRESS_CUDA_TRY(cudaEventCreate(&e1));
    struct EvGuard {
        cudaEvent_t a, b;
        ~EvGuard() { cudaEventDestroy(a); cudaEventDestroy(b); }
    } guard{e0, e1};
    const double setup_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    DRESS_CUDA_TRY(cudaEventRecord(e0, st));
    if (one_cta) {
        DRESS_TRY(launch_batch(L, ctx.num_sms, st));
    } else {
        Status ls = launch_cluster_fit(L.parents, E, N, lnc, ctx.num_sms, st);
        if (ls.code == DRESSX_EUNSUPPORTED) return Status::Ok();     // the multi-kernel fit takes it
        DRESS_TRY(ls);
    }
    DRESS_CUDA_TRY(cudaEventRecord(e1, st));

    // statistics and results come back in one copy through the stage
    DRESS_CUDA_TRY(counted_memcpy(h + off_stats, dv + off_stats, total - off_stats, cudaMemcpyDeviceToHost, st));
    DRESS_CUDA_TRY(cudaStreamSynchronize(st));
    unsigned long long sv[ST_WORDS];
    std::memcpy(sv, h + off_stats, sizeof sv);
    std::memcpy(g->edge_dress, h + off_vals, (size_t)E * sizeof(double));
    // the norms of the last sweep (none without sweeps), as fit_graph leaves them
    if (sv[ST_SWEEPS] > 0) std::memcpy(g->vertex_dress, h + off_vals + (size_t)E * sizeof(double), (size_t)N * sizeof(double));
    float it_ms = 0.f;
    cudaEventElapsedTime(&it_ms, e0, e1);
    if (iterations) *iterations = (int)(long long)sv[ST_ITERATIONS];
    if (delta && sv[ST_SWEEPS] > 0) std::memcpy(delta, &sv[ST_DELTA], sizeof(double));
    if (stats) {
        *stats = FitStats{};
        stats->T = T;
        stats->sweeps = (int)sv[ST_SWEEPS];
        stats->setup_ms = setup_ms;
        stats->iterate_ms = it_ms;
    }
    used = true;
    return Status::Ok();
}

}  // namespace dress
