// fit_graph.cu -- single-graph DRESS fit on one B200 (dress_fit_cuda).
//
// Reference behaviour: libdress/src/dress.c:546-608 (sequential fit) and the
// slot it fills, libdress/src/cuda/dress_cuda.cu:445-707.
//
// Layout in HBM (all built on the device from the caller's CSR):
//   * common-neighbour tables: for every edge e=(u,v) the list of edge-id
//     pairs (e_ux, e_vx), x in N[u] n N[v].  UNDIRECTED simple graphs get them
//     from degree-ordered triangle listing (each triangle found once from its
//     lowest-rank vertex); other variants and multigraphs from the
//     reference's exact merge walk per edge; graphs built with
//     precompute_intercepts reuse their own tables.
//   * vertices and edges are renumbered so that items with the same number of
//     sum terms are contiguous ("bins": 1, 2, 4, 8, 16, 32 terms -> one thread
//     per item with a register sorting network; <=1024 -> one warp per item
//     with a shared-memory sort; more -> one block per item).  Renumbering
//     makes every per-edge stream (endpoints, weight, value, next value)
//     sequential and packs the edges that appear in triangles -- the only ones
//     gathered by the edge sweep -- into one L2-sized region at the end.
//   * p = w*d is stored next to d (double-buffered) for weighted graphs, so a
//     term costs one gather; for uniform weights p is formed on the fly.
// Each sweep is one vertex-norm pass and one edge pass per bin; the edge pass
// folds max|d_next - d| into a per-sweep slot, and every kernel of sweep i
// returns at once if sweep i-1 already met the tolerance, so a chunk of
// sweeps is launched back to back and the host reads the slots once per chunk.
#include <algorithm>
#include <climits>
#include <chrono>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

#include "common.cuh"
#include "engine.h"
#include "hist.h"
#include "sweep.cuh"

namespace dress {
namespace {

constexpr int MAX_CHUNK = 32;      // sweeps launched per host check (<= RING/2)
constexpr int LOCALITY_MIN_EDGES = 1 << 20;   // graphs renumbered for gather locality
using namespace sweep;

__device__ __forceinline__ unsigned lanemask_lt()
{
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// ------------------------------------------------------------------------
// set-up kernels
// ------------------------------------------------------------------------

// flags[0]: malformed input, flags[1]: a row repeats a neighbour,
// flags[2]: edge weights are not all bit-identical, flags[3]: max row length.
// One warp per row (a hub's row is spread over the lanes).  A row outside
// [0, S) or with end < begin is flagged and not read, so a malformed
// adj_offset never leads to a read outside adj_target.
__global__ void k_validate_rows(int N, int E, long long S, const int *off, const int *tgt, const int *eidx,
                                int *deg, int *flags)
{
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    int rmax = 0, bad = 0, dup = 0;
    for (int u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < N; u += nw) {
        const long long b = off[u], e = off[u + 1];
        if (e < b || b < 0 || e > S) {
            bad |= 1;
            if (lane == 0) deg[u] = 0;
            continue;
        }
        if (lane == 0) deg[u] = (int)(e - b);
        rmax = max(rmax, (int)(e - b));
        for (long long q = b + lane; q < e; q += 32) {
            const int x = tgt[q], ei = eidx[q];
            if (x < 0 || x >= N || ei < 0 || ei >= E) bad |= 2;
            if (q > b) {
                const int prev = tgt[q - 1];
                if (x == prev) dup = 1;
                else if (x < prev) bad |= 4;
            }
        }
    }
    rmax = __reduce_max_sync(0xffffffffu, rmax);
    bad = __reduce_or_sync(0xffffffffu, bad);
    dup = __reduce_or_sync(0xffffffffu, dup);
    if (lane == 0) {
        if (bad) atomicOr(&flags[0], bad);
        if (dup) flags[1] = 1;
        if (rmax) atomicMax(&flags[3], rmax);
    }
}
__global__ void k_validate_edges(int N, int E, const int *U, const int *V, const double *w, int *flags)
{
    unsigned long long w0 = E > 0 ? (unsigned long long)__double_as_longlong(w[0]) : 0ULL;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += gridDim.x * blockDim.x) {
        int u = U[e], v = V[e];
        if (u < 0 || u >= N || v < 0 || v >= N) atomicOr(&flags[0], 8);
        if ((unsigned long long)__double_as_longlong(w[e]) != w0) flags[2] = 1;
    }
}

// ---- intercepts from the graph's own tables ----
__global__ void k_given_counts(int E, const int *io, int *cnt, int *flags)
{
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += gridDim.x * blockDim.x) {
        int c = io[e + 1] - io[e];
        if (c < 0) { atomicOr(&flags[0], 16); c = 0; }
        cnt[e] = c;
    }
}

__global__ void k_given_pairs(int E, const int *io, const int *ux, const int *vx,
                              const long long *ioff, int2 *pairs, int *flags)
{
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += gridDim.x * blockDim.x) {
        long long o = ioff[e];
        int b = io[e], n = io[e + 1] - b;
        for (int k = 0; k < n; ++k) {
            int a = ux[b + k], c = vx[b + k];
            if (a < 0 || a >= E || c < 0 || c >= E) { atomicOr(&flags[0], 32); a = c = e; }
            pairs[o + k] = make_int2(a, c);
        }
    }
}

// ---- intercepts by the reference's merge walk (any variant, multigraphs) ----
template <bool FILL>
__global__ void k_merge_intercepts(int E, const int *U, const int *V, const int *off, const int *tgt,
                                   const int *eidx, int *cnt, const long long *ioff, int2 *pairs)
{
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += gridDim.x * blockDim.x) {
        int iu = off[U[e]], iu_end = off[U[e] + 1];
        int iv = off[V[e]], iv_end = off[V[e] + 1];
        long long o = FILL ? ioff[e] : 0;
        int c = 0;
        while (iu < iu_end && iv < iv_end) {
            int x = tgt[iu], y = tgt[iv];
            if (x == y) {
                if (FILL) pairs[o + c] = make_int2(eidx[iu], eidx[iv]);
                ++c;
            }
            iu += (x <= y);
            iv += (x >= y);
        }
        if (!FILL) cnt[e] = c;
    }
}

// ---- intercepts by degree-ordered triangle listing (UNDIRECTED, simple) ----
__device__ __forceinline__ unsigned long long rank_key(const int *deg, int v)
{
    return ((unsigned long long)(unsigned)deg[v] << 32) | (unsigned)v;
}

// The oriented rows: the neighbours of higher (degree, id) rank, in row
// order (ascending id).  One warp per row; the fill compacts by ballot.
__global__ void k_orient_count(int N, const int *off, const int *tgt, const int *deg, int *ocnt)
{
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < N; u += nw) {
        const unsigned long long ku = rank_key(deg, u);
        int c = 0;
        for (int q = off[u] + lane; q < off[u + 1]; q += 32) c += rank_key(deg, tgt[q]) > ku;
        c = __reduce_add_sync(0xffffffffu, c);
        if (lane == 0) ocnt[u] = c;
    }
}
__global__ void k_orient_fill(int N, const int *off, const int *tgt, const int *eidx, const int *deg,
                              const long long *ooff, int *otgt, int *oeid, int *osrc)
{
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < N; u += nw) {
        const unsigned long long ku = rank_key(deg, u);
        long long o = ooff[u];
        const int b = off[u], e = off[u + 1];
        for (int q0 = b; q0 < e; q0 += 32) {
            const int q = q0 + lane;
            int x = 0;
            bool keep = false;
            if (q < e) {
                x = tgt[q];
                keep = rank_key(deg, x) > ku;
            }
            const unsigned m = __ballot_sync(0xffffffffu, keep);
            if (keep) {
                const long long at = o + __popc(m & lanemask_lt());
                otgt[at] = x;
                oeid[at] = eidx[q];
                osrc[at] = u;
            }
            o += __popc(m);
        }
    }
}

// Each oriented edge a->b intersects out(a) with out(b) (both ascending by id).
// A common c closes the triangle {a,b,c}; each of its three edges receives
// the pair of the other two (the order inside a pair is irrelevant: the term
// is their sum).
// The pairs an oriented edge finds for itself go to the head of its own list
// (own[eab] of them, counted in the first pass), without atomics; the pairs
// it finds for its triangles' other two edges go through their cursors,
// which start after those heads.  Two rows of very different lengths are
// intersected by binary searches of the short row's ids in the long one
// (a merge walk would step through the whole long row).
template <bool FILL>
__global__ void k_triangles(long long M, const long long *ooff, const int *otgt, const int *oeid,
                            const int *osrc, int *cnt, int *own_cnt, const long long *ioff,
                            unsigned long long *cursor, int2 *pairs)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < M;
         q += (long long)gridDim.x * blockDim.x) {
        int a = osrc[q], b = otgt[q], eab = oeid[q];
        long long pa = ooff[a], pa_end = ooff[a + 1];
        long long pb = ooff[b], pb_end = ooff[b + 1];
        int own = 0;                           // this edge's triangles so far
        const long long head = FILL ? ioff[eab] : 0;
        auto found = [&](int eac, int ebc) {
            if (!FILL) {
                ++own;
                atomicAdd(&cnt[eac], 1);
                atomicAdd(&cnt[ebc], 1);
            } else {
                pairs[head + own++] = make_int2(eac, ebc);
                pairs[atomicAdd(&cursor[eac], 1ULL)] = make_int2(eab, ebc);
                pairs[atomicAdd(&cursor[ebc], 1ULL)] = make_int2(eab, eac);
            }
        };
        const long long la = pa_end - pa, lb = pb_end - pb;
        const long long ls = la < lb ? la : lb, ll = la < lb ? lb : la;
        if (ls > 0 && ls * (64 - __clzll(ll)) < ll) {
            const bool a_short = la <= lb;
            const long long s0 = a_short ? pa : pb, s1 = a_short ? pa_end : pb_end;
            long long lo = a_short ? pb : pa;
            const long long l1 = a_short ? pb_end : pa_end;
            for (long long i = s0; i < s1 && lo < l1; ++i) {
                const int x = otgt[i];
                long long L = lo, R = l1;              // first id >= x in the long row
                while (L < R) {
                    const long long mid = (L + R) >> 1;
                    if (otgt[mid] < x) L = mid + 1;
                    else R = mid;
                }
                lo = L;
                if (L < l1 && otgt[L] == x) {
                    found(oeid[a_short ? i : L], oeid[a_short ? L : i]);
                    ++lo;
                }
            }
        } else {
            while (pa < pa_end && pb < pb_end) {
                int x = otgt[pa], y = otgt[pb];
                if (x == y) {
                    found(oeid[pa], oeid[pb]);
                    ++pa;
                    ++pb;
                } else if (x < y) {
                    ++pa;
                } else {
                    ++pb;
                }
            }
        }
        if (!FILL) {
            own_cnt[eab] = own;                // each edge is one oriented edge
            if (own) atomicAdd(&cnt[eab], own);
        }
    }
}

// each edge's cursor: the start of its pair list past its own pairs
__global__ void k_cursor_init(long long n, const long long *ioff, const int *own_cnt, unsigned long long *cursor)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        cursor[i] = (unsigned long long)(ioff[i] + own_cnt[i]);
}

// ---- binning (terms per item) and renumbering ----
__global__ void k_bin_count(int n, const int *len, int *bin_cnt)
{
    __shared__ int sc[NF];
    for (int f = threadIdx.x; f < NF; f += blockDim.x) sc[f] = 0;
    __syncthreads();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        atomicAdd(&sc[fine_of((long long)len[i])], 1);
    __syncthreads();
    for (int f = threadIdx.x; f < NF; f += blockDim.x)
        if (sc[f]) atomicAdd(&bin_cnt[f], sc[f]);
}

// stored terms per coarse bin
__global__ void k_bin_terms(int n, const int *len, unsigned long long *terms)
{
    __shared__ unsigned long long sc[NB];
    if (threadIdx.x < NB) sc[threadIdx.x] = 0;
    __syncthreads();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        atomicAdd(&sc[bin_of((long long)len[i])], (unsigned long long)len[i]);
    __syncthreads();
    if (threadIdx.x < NB && sc[threadIdx.x]) atomicAdd(&terms[threadIdx.x], sc[threadIdx.x]);
}

// Scatter items to their fine keys' ranges; lanes of a warp that share a key
// take consecutive slots (one atomic per group), which keeps neighbouring
// items neighbours.
__global__ void k_bin_scatter(int n, const int *len, int *cursor, int *perm, int *inv)
{
    int lane = threadIdx.x & 31;
    for (int i0 = blockIdx.x * blockDim.x; i0 < n; i0 += gridDim.x * blockDim.x) {
        int i = i0 + threadIdx.x;
        unsigned active = __ballot_sync(0xffffffffu, i < n);
        if (i < n) {
            int b = fine_of((long long)len[i]);
            unsigned peers = __match_any_sync(active, b);
            int leader = __ffs(peers) - 1;
            int base = 0;
            if (lane == leader) base = atomicAdd(&cursor[b], __popc(peers));
            base = __shfl_sync(peers, base, leader);
            int pos = base + __popc(peers & lanemask_lt());
            perm[pos] = i;
            inv[i] = pos;
        }
    }
}

// Sort keys of the edge renumbering of a large graph: the edges without
// common neighbours first, then the others; within each part by owner -- the
// endpoint of lower (degree, id) rank, the triangle listing's orientation --
// in the new vertex numbering, then by the other endpoint.  A vertex owns
// most edges of its row unless it is a hub, so a row's edges sit in two runs
// and the (u, x) edges of an edge's common-neighbour pairs next to each
// other: neighbouring lanes gather neighbouring products.
// vb: bits of a vertex id (the keys take 2 vb + 1 bits, so the radix sort
// skips the passes over their zero high bytes)
__global__ void k_edge_keys(int E, const int *U, const int *V, const int *deg, const int *vinv, const int *cnt,
                            int vb, unsigned long long *keys, unsigned *vals)
{
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += gridDim.x * blockDim.x) {
        const int u = U[e], v = V[e];
        const bool uo = rank_key(deg, u) <= rank_key(deg, v);
        const unsigned long long o = (unsigned)vinv[uo ? u : v], x = (unsigned)vinv[uo ? v : u];
        keys[e] = ((unsigned long long)(cnt[e] > 0) << (2 * vb)) | (o << vb) | x;
        vals[e] = (unsigned)e;
    }
}

// size class of an edge with n > 0 common-neighbour pairs (the order of the
// edge lists, see sweep::EdgeClasses)
__device__ __forceinline__ unsigned pair_class(int n)
{
    return n <= 16 ? 0u : n <= 64 ? 3u : n <= 256 ? 2u : n <= MED_CAP ? 1u : n <= BIG_CAP ? 4u : 5u;
}

__global__ void k_class_keys(int e0, int E, const int *ncnt, unsigned long long *keys, unsigned *vals)
{
    for (int j = e0 + blockIdx.x * blockDim.x + threadIdx.x; j < E; j += gridDim.x * blockDim.x) {
        keys[j - e0] = pair_class(ncnt[j]);    // stable sort: ids stay ascending per class
        vals[j - e0] = (unsigned)j;
    }
}

// bounds[c] = first position of class c in the sorted keys (c = 0..6)
__global__ void k_class_bounds(int n, const unsigned long long *keys, int *bounds)
{
    const int c = threadIdx.x;
    if (c > 6) return;
    const unsigned long long want = (unsigned long long)c;
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (keys[mid] < want) lo = mid + 1;
        else hi = mid;
    }
    bounds[c] = lo;
}

__global__ void k_iota(int n, int base, int *out)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = base + i;
}

__global__ void k_inverse(int n, const unsigned *perm, int *pinv, int *inv)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        pinv[i] = (int)perm[i];
        inv[perm[i]] = i;
    }
}

// Each edge's pairs put in (first, second) edge-id order, in place: a
// warp's lanes then gather neighbouring products (an owner's edges are
// contiguous).  The order only serves locality -- the certified sums give the
// same bits in any order -- so edges past BIG_CAP pairs keep theirs.
__device__ __forceinline__ unsigned long long pair_word(int2 pr)
{
    return ((unsigned long long)(unsigned)pr.x << 32) | (unsigned)pr.y;
}
__device__ __forceinline__ int2 word_pair(unsigned long long w)
{
    return make_int2((int)(unsigned)(w >> 32), (int)(unsigned)w);
}

// up to 16 pairs: one thread per edge, insertion sort
__global__ void k_sort_pairs_thr(const int *list, int begin, int end, const long long *ioff, int2 *pairs)
{
    for (int x = begin + blockIdx.x * blockDim.x + threadIdx.x; x < end; x += gridDim.x * blockDim.x) {
        const int j = list[x];
        const long long b = ioff[j];
        const int n = (int)(ioff[j + 1] - b);
        unsigned long long w[16];
        for (int k = 0; k < n && k < 16; ++k) {
            const unsigned long long t = pair_word(pairs[b + k]);
            int i = k;
            for (; i > 0 && w[i - 1] > t; --i) w[i] = w[i - 1];
            w[i] = t;
        }
        for (int k = 0; k < n && k < 16; ++k) pairs[b + k] = word_pair(w[k]);
    }
}

// bitonic sort of buf[0, P) (P a power of two) by `nt` cooperating threads
template <bool BLOCK>
__device__ __forceinline__ void bitonic(unsigned long long *buf, int P, int tid, int nt)
{
    for (int k = 2; k <= P; k <<= 1)
        for (int h = k >> 1; h > 0; h >>= 1) {
            for (int i = tid; i < P; i += nt) {
                const int o = i ^ h;
                if (o > i) {
                    const unsigned long long a = buf[i], c = buf[o];
                    if ((a > c) == ((i & k) == 0)) {
                        buf[i] = c;
                        buf[o] = a;
                    }
                }
            }
            if (BLOCK) __syncthreads();
            else __syncwarp();
        }
}

constexpr int SORT_WARP_CAP = MED_CAP;     // pairs a warp sorts in shared memory
constexpr int SORT_WARPS = 8;

// 17..MED_CAP pairs: one warp per edge
__global__ void __launch_bounds__(32 * SORT_WARPS) k_sort_pairs_warp(const int *list, int begin, int end,
                                                                    const long long *ioff, int2 *pairs)
{
    __shared__ unsigned long long sb[SORT_WARPS][SORT_WARP_CAP];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    unsigned long long *buf = sb[wid];
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int x = begin + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); x < end; x += nw) {
        const int j = list[x];
        const long long b = ioff[j];
        const int n = (int)(ioff[j + 1] - b);
        if (n > SORT_WARP_CAP) continue;
        int P = 32;
        while (P < n) P <<= 1;
        for (int k = lane; k < P; k += 32) buf[k] = k < n ? pair_word(pairs[b + k]) : ~0ULL;
        __syncwarp();
        bitonic<false>(buf, P, lane, 32);
        for (int k = lane; k < n; k += 32) pairs[b + k] = word_pair(buf[k]);
        __syncwarp();
    }
}

constexpr int SORT_BLK_THR = 512;

// MED_CAP+1..BIG_CAP pairs: one block per edge
__global__ void __launch_bounds__(SORT_BLK_THR) k_sort_pairs_blk(const int *list, int begin, int end,
                                                                 const long long *ioff, int2 *pairs)
{
    __shared__ unsigned long long buf[BIG_CAP];
    for (int x = begin + (int)blockIdx.x; x < end; x += gridDim.x) {
        const int j = list[x];
        const long long b = ioff[j];
        const int n = (int)(ioff[j + 1] - b);
        if (n > BIG_CAP) continue;
        int P = 32;
        while (P < n) P <<= 1;
        for (int k = threadIdx.x; k < P; k += blockDim.x) buf[k] = k < n ? pair_word(pairs[b + k]) : ~0ULL;
        __syncthreads();
        bitonic<true>(buf, P, threadIdx.x, blockDim.x);
        for (int k = threadIdx.x; k < n; k += blockDim.x) pairs[b + k] = word_pair(buf[k]);
        __syncthreads();
    }
}

// Each row's slots in edge-id order, in place, so that a vertex's owned
// edges (one contiguous id run each in the two edge parts) are neighbouring
// slots: their gathers in the vertex phase read neighbouring products.  Rows
// of vertices [lo, hi), which all have n slots of one size class; rows past
// BIG_CAP slots keep their order.
__global__ void k_sort_rows_thr(int lo, int hi, const long long *row_off, int *row_eid)
{
    for (int i = lo + blockIdx.x * blockDim.x + threadIdx.x; i < hi; i += gridDim.x * blockDim.x) {
        const long long b = row_off[i];
        const int n = (int)(row_off[i + 1] - b);
        int w[16];
        for (int k = 0; k < n && k < 16; ++k) {
            const int t = row_eid[b + k];
            int j = k;
            for (; j > 0 && w[j - 1] > t; --j) w[j] = w[j - 1];
            w[j] = t;
        }
        for (int k = 0; k < n && k < 16; ++k) row_eid[b + k] = w[k];
    }
}

__global__ void __launch_bounds__(32 * SORT_WARPS) k_sort_rows_warp(int lo, int hi, const long long *row_off,
                                                                    int *row_eid)
{
    __shared__ unsigned long long sb[SORT_WARPS][SORT_WARP_CAP];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    unsigned long long *buf = sb[wid];
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int i = lo + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); i < hi; i += nw) {
        const long long b = row_off[i];
        const int n = (int)(row_off[i + 1] - b);
        if (n > SORT_WARP_CAP) continue;
        int P = 32;
        while (P < n) P <<= 1;
        for (int k = lane; k < P; k += 32) buf[k] = k < n ? (unsigned long long)(unsigned)row_eid[b + k] : ~0ULL;
        __syncwarp();
        bitonic<false>(buf, P, lane, 32);
        for (int k = lane; k < n; k += 32) row_eid[b + k] = (int)(unsigned)buf[k];
        __syncwarp();
    }
}

__global__ void __launch_bounds__(SORT_BLK_THR) k_sort_rows_blk(int lo, int hi, const long long *row_off, int *row_eid)
{
    __shared__ unsigned long long buf[BIG_CAP];
    for (int i = lo + (int)blockIdx.x; i < hi; i += gridDim.x) {
        const long long b = row_off[i];
        const int n = (int)(row_off[i + 1] - b);
        if (n > BIG_CAP) continue;
        int P = 32;
        while (P < n) P <<= 1;
        for (int k = threadIdx.x; k < P; k += blockDim.x)
            buf[k] = k < n ? (unsigned long long)(unsigned)row_eid[b + k] : ~0ULL;
        __syncthreads();
        bitonic<true>(buf, P, threadIdx.x, blockDim.x);
        for (int k = threadIdx.x; k < n; k += blockDim.x) row_eid[b + k] = (int)(unsigned)buf[k];
        __syncthreads();
    }
}

__global__ void k_gather_seg(int n, const int *perm, const int *len, int *out)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = len[perm[i]];
}

__global__ void k_fix_inv(int n, int base, const int *perm, int *inv)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) inv[perm[base + i]] = base + i;
}

__global__ void k_gather_deg(int N, const int *vperm, const int *deg, int *ndeg)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
        ndeg[i] = deg[vperm[i]];
}

// one warp per (renumbered) vertex: copy its row with renumbered edge ids
__global__ void k_new_rows(int N, const int *vperm, const int *off, const int *eidx, const int *einv,
                           const long long *row_off, int *row_eid, const double *nw_in, double *nw_out)
{
    int lane = threadIdx.x & 31;
    int warps = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < N; i += warps) {
        int u = vperm[i];
        int b = off[u], n = off[u + 1] - b;
        long long o = row_off[i];
        for (int k = lane; k < n; k += 32) row_eid[o + k] = einv[eidx[b + k]];
        if (lane == 0) nw_out[i] = nw_in[u];
    }
}

__global__ void k_new_edges(int E, const int *eperm, const int *U, const int *V, const int *vinv,
                            const double *w, const double *d, const int *cnt, int *eu, int *ev,
                            double *wn, double *d0, double *p0, int *ncnt)
{
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < E; j += gridDim.x * blockDim.x) {
        int e = eperm[j];
        eu[j] = vinv[U[e]];
        ev[j] = vinv[V[e]];
        double we = w[e], de = d[e];
        d0[j] = de;
        if (wn) { wn[j] = we; p0[j] = dmul(we, de); }
        ncnt[j] = cnt[e];
    }
}

// The pairs of the edges in list[lo, hi), copied to their new places with
// the new edge ids: GW lanes per edge (1 for the short classes, a warp for
// edges of 17 pairs or more, so a long edge is not one thread's loop).
template <int GW>
__global__ void k_new_pairs(const int *list, int lo, int hi, const int *eperm, const long long *ioff_old,
                            const int2 *pairs_old, const int *einv, const long long *ioff_new, int2 *pairs_new)
{
    const int lane = threadIdx.x & (GW - 1);
    const long long ng = ((long long)gridDim.x * blockDim.x) / GW;
    for (long long x = lo + (blockIdx.x * (long long)blockDim.x + threadIdx.x) / GW; x < hi; x += ng) {
        const int j = list[x], e = eperm[j];
        const long long a = ioff_old[e], n = ioff_old[e + 1] - a, o = ioff_new[j];
        for (long long k = lane; k < n; k += GW) {
            const int2 pr = pairs_old[a + k];
            pairs_new[o + k] = make_int2(einv[pr.x], einv[pr.y]);
        }
    }
}

__global__ void k_fill(int n, double v, double *out)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = v;
}

__global__ void k_unpermute(int n, const int *perm, const double *src, double *dst)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        dst[perm[i]] = src[i];
}

// An upload on a host thread of its own, through the context's second stage
// on stream side2: started before the kernels that need only the CSR, joined
// before the first that reads its arrays.  The destructor joins, so no early
// return leaves the thread running.
struct BackgroundUpload {
    std::thread th;
    Status result;
    bool running = false;
    double wait_ms = 0.0;                  // time the caller spent blocked in join()
    Status start(std::vector<HostSpan> spans, const Ctx &ctx)
    {
        // the destination buffers were allocated in stream order on ctx.st
        DRESS_CUDA_TRY(cudaEventRecord(ctx.fork, ctx.st));
        DRESS_CUDA_TRY(cudaStreamWaitEvent(ctx.side2, ctx.fork, 0));
        try {
            th = std::thread([this, sp = std::move(spans), &ctx]() {
                const cudaError_t e = cudaSetDevice(ctx.device);
                if (e != cudaSuccess) {
                    result = Status::Err(DRESSX_ECUDA, cudaGetErrorString(e));
                    return;
                }
                result = staged_upload_via(sp.data(), (int)sp.size(), ctx.stage2, ctx.side2);
            });
        } catch (...) {
            return Status::Err(DRESSX_ENOMEM, "cannot start the upload thread");
        }
        running = true;
        return Status::Ok();
    }
    Status join()
    {
        if (running) {
            const auto w0 = std::chrono::steady_clock::now();
            th.join();
            running = false;
            wait_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - w0).count();
        }
        return result;
    }
    ~BackgroundUpload()
    {
        if (running) th.join();
    }
};

double ms_since(std::chrono::steady_clock::time_point t0)
{
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

Status fit_graph(p_dress_graph_t g, int max_iterations, double epsilon, int *iterations,
                 double *delta, FitStats *stats, const Ctx &ctx)
{
    auto t0 = std::chrono::steady_clock::now();
    if (!g) return Status::Err(DRESSX_EINVAL, "graph is NULL");
    const int N = g->N, E = g->E;
    if (N < 0 || E < 0) return Status::Err(DRESSX_EINVAL, "negative N or E");
    if (max_iterations <= 0) {                       // reference: loop body never runs
        if (iterations) *iterations = max_iterations;
        return Status::Ok();
    }
    if (N > 0 && (!g->adj_offset || !g->vertex_dress))
        return Status::Err(DRESSX_EINVAL, "graph has NULL vertex arrays");
    if (E > 0 && (!g->U || !g->V || !g->edge_weight || !g->edge_dress || !g->adj_target ||
                  !g->adj_edge_idx))
        return Status::Err(DRESSX_EINVAL, "graph has NULL edge arrays");
    const long long S = N > 0 ? g->adj_offset[N] : 0;
    if (N > 0 && (g->adj_offset[0] != 0 || S < 0)) return Status::Err(DRESSX_EINVAL, "bad adj_offset");
    {
        // small graphs: the whole fit in one launch
        bool used = false;
        DRESS_TRY(fit_small(g, max_iterations, epsilon, iterations, delta, stats, ctx, used));
        if (used) return Status::Ok();
    }

    cudaStream_t st = ctx.st;
    const int sms = ctx.num_sms;
    const int fwd = (g->variant == DRESS_VARIANT_FORWARD || g->variant == DRESS_VARIANT_BACKWARD);

    // ---- upload: the CSR first; the edge arrays on a host thread of their
    // own, beside the row validation and the triangle listing (CSR only) --------
    DevBuf<int> d_off, d_tgt, d_eidx, d_U, d_V;
    DevBuf<double> d_w, d_d, d_nw;
    DRESS_TRY(d_off.alloc((size_t)N + 1, st));
    DRESS_TRY(d_tgt.alloc((size_t)S, st));
    DRESS_TRY(d_eidx.alloc((size_t)S, st));
    DRESS_TRY(d_U.alloc((size_t)E, st));
    DRESS_TRY(d_V.alloc((size_t)E, st));
    DRESS_TRY(d_w.alloc((size_t)E, st));
    DRESS_TRY(d_d.alloc((size_t)E, st));
    DRESS_TRY(d_nw.alloc((size_t)N, st));
    {
        const HostSpan csr[3] = {{g->adj_offset, d_off.get(), ((size_t)N + 1) * sizeof(int)},
                                 {g->adj_target, d_tgt.get(), (size_t)S * sizeof(int)},
                                 {g->adj_edge_idx, d_eidx.get(), (size_t)S * sizeof(int)}};
        DRESS_TRY(staged_upload(csr, 3, ctx));
    }
    BackgroundUpload edge_up;
    {
        std::vector<HostSpan> spans = {{g->U, d_U.get(), (size_t)E * sizeof(int)},
                                       {g->V, d_V.get(), (size_t)E * sizeof(int)},
                                       {g->edge_weight, d_w.get(), (size_t)E * sizeof(double)},
                                       {g->edge_dress, d_d.get(), (size_t)E * sizeof(double)}};
        if (g->NW) spans.push_back({g->NW, d_nw.get(), (size_t)N * sizeof(double)});
        DRESS_TRY(edge_up.start(std::move(spans), ctx));
    }
    const double t_upload = ms_since(t0);
    if (!g->NW && N)                           // NULL vertex weights mean all 1.0
        count_launch(), k_fill<<<grid_for(N, 256, 16 * sms), 256, 0, st>>>(N, 1.0, d_nw.get());

    // ---- validate the rows ---------------------------------------------------
    DevBuf<int> d_flags, d_deg, d_cnt;
    DRESS_TRY(d_flags.alloc(8, st));
    DRESS_TRY(d_deg.alloc((size_t)N, st));
    DRESS_TRY(d_cnt.alloc((size_t)E, st));
    DRESS_CUDA_TRY(cudaMemsetAsync(d_flags.get(), 0, 8 * sizeof(int), st));
    count_launch(), k_validate_rows<<<grid_for((long long)N * 32, 256, 16 * sms), 256, 0, st>>>(
        N, E, S, d_off.get(), d_tgt.get(), d_eidx.get(), d_deg.get(), d_flags.get());
    DRESS_CUDA_TRY(cudaGetLastError());
    int flags[8];
    DRESS_CUDA_TRY(counted_memcpy(flags, d_flags.get(), sizeof(flags), cudaMemcpyDeviceToHost, st));
    DRESS_CUDA_TRY(cudaStreamSynchronize(st));
    double t_valid = ms_since(t0) - t_upload;
    if (flags[0]) return Status::Err(DRESSX_EINVAL, "malformed graph (CSR or edge endpoints out of range)");
    const bool dup = flags[1] != 0;
    const long long max_row = flags[3];
    const double wc = E > 0 ? g->edge_weight[0] : 1.0;
    // The edge arrays, validated once they are on the device: before the
    // pairs unless the triangle listing (CSR only) makes them.
    bool uniform = true;
    auto validate_edges = [&]() -> Status {
        DRESS_TRY(edge_up.join());
        const auto v0 = std::chrono::steady_clock::now();
        count_launch(), k_validate_edges<<<grid_for(E, 256, 16 * sms), 256, 0, st>>>(N, E, d_U.get(), d_V.get(),
                                                                                      d_w.get(), d_flags.get());
        DRESS_CUDA_TRY(cudaGetLastError());
        DRESS_CUDA_TRY(counted_memcpy(flags, d_flags.get(), sizeof(flags), cudaMemcpyDeviceToHost, st));
        DRESS_CUDA_TRY(cudaStreamSynchronize(st));
        t_valid += ms_since(v0);
        if (flags[0]) return Status::Err(DRESSX_EINVAL, "malformed graph (CSR or edge endpoints out of range)");
        uniform = flags[2] == 0;
        return Status::Ok();
    };
    const bool tri_path = !(g->precompute_intercepts && g->intercept_offset) &&
                          g->variant == DRESS_VARIANT_UNDIRECTED && !dup;
    if (!tri_path) DRESS_TRY(validate_edges());

    // ---- common-neighbour tables (original edge ids) -------------------------
    DevBuf<long long> d_ioff_old, d_scan_tmp;
    DevBuf<int2> d_pairs_old;
    // the oriented rows of the triangle listing, alive until its fill is joined
    DevBuf<int> d_ocnt, d_otgt, d_oeid, d_osrc, d_own;
    DevBuf<long long> d_ooff;
    DevBuf<unsigned long long> d_cursor;
    // Declared after the buffers the side-stream fill reads, so that on an
    // early return it waits for the fill before they are freed.
    struct SideFill {
        cudaStream_t side;
        bool pending = false;
        ~SideFill()
        {
            if (pending) cudaStreamSynchronize(side);
        }
    } fill{ctx.side};
    DRESS_TRY(d_ioff_old.alloc((size_t)E + 1, st));
    DRESS_TRY(d_scan_tmp.alloc(scan_tmp_elems((long long)(S > E ? S : E) + N + 1), st));
    long long T = 0;
    const int eg = (int)grid_for(E, 256, 32 * sms);
    if (g->precompute_intercepts && g->intercept_offset) {
        DevBuf<int> d_io, d_ux, d_vx;
        long long Tg = g->intercept_offset[E];
        if (Tg < 0) return Status::Err(DRESSX_EINVAL, "bad intercept_offset");
        DRESS_TRY(d_io.alloc((size_t)E + 1, st));
        DRESS_TRY(d_ux.alloc((size_t)Tg, st));
        DRESS_TRY(d_vx.alloc((size_t)Tg, st));
        const HostSpan spans[3] = {{g->intercept_offset, d_io.get(), ((size_t)E + 1) * sizeof(int)},
                                   {g->intercept_edge_ux, d_ux.get(), (size_t)Tg * sizeof(int)},
                                   {g->intercept_edge_vx, d_vx.get(), (size_t)Tg * sizeof(int)}};
        DRESS_TRY(staged_upload(spans, 3, ctx));
        count_launch(), k_given_counts<<<eg, 256, 0, st>>>(E, d_io.get(), d_cnt.get(), d_flags.get());
        DRESS_TRY(exclusive_scan_i32(d_cnt.get(), d_ioff_old.get(), E, d_scan_tmp.get(), st));
        DRESS_CUDA_TRY(counted_memcpy(&T, d_ioff_old.get() + E, sizeof(T), cudaMemcpyDeviceToHost, st));
        DRESS_CUDA_TRY(cudaStreamSynchronize(st));
        DRESS_TRY(d_pairs_old.alloc((size_t)(T > 0 ? T : 1), st));
        count_launch(), k_given_pairs<<<eg, 256, 0, st>>>(E, d_io.get(), d_ux.get(), d_vx.get(), d_ioff_old.get(),
                                          d_pairs_old.get(), d_flags.get());
    } else if (g->variant == DRESS_VARIANT_UNDIRECTED && !dup) {
        DRESS_TRY(d_ocnt.alloc((size_t)N, st));
        DRESS_TRY(d_ooff.alloc((size_t)N + 1, st));
        DRESS_TRY(d_otgt.alloc((size_t)(S > 0 ? S : 1), st));
        DRESS_TRY(d_oeid.alloc((size_t)(S > 0 ? S : 1), st));
        DRESS_TRY(d_osrc.alloc((size_t)(S > 0 ? S : 1), st));
        const int vg = (int)grid_for((long long)N * 32, 256, 32 * sms);     // a warp per row
        count_launch(), k_orient_count<<<vg, 256, 0, st>>>(N, d_off.get(), d_tgt.get(), d_deg.get(), d_ocnt.get());
        DRESS_TRY(exclusive_scan_i32(d_ocnt.get(), d_ooff.get(), N, d_scan_tmp.get(), st));
        count_launch(), k_orient_fill<<<vg, 256, 0, st>>>(N, d_off.get(), d_tgt.get(), d_eidx.get(), d_deg.get(),
                                          d_ooff.get(), d_otgt.get(), d_oeid.get(), d_osrc.get());
        long long M = 0;
        DRESS_CUDA_TRY(counted_memcpy(&M, d_ooff.get() + N, sizeof(M), cudaMemcpyDeviceToHost, st));
        DRESS_CUDA_TRY(cudaMemsetAsync(d_cnt.get(), 0, (size_t)E * sizeof(int), st));
        DRESS_CUDA_TRY(cudaStreamSynchronize(st));
        const int tg = (int)grid_for(M, 256, 64 * sms);
        DRESS_TRY(d_own.alloc((size_t)(E > 0 ? E : 1), st));
        DRESS_CUDA_TRY(cudaMemsetAsync(d_own.get(), 0, (size_t)E * sizeof(int), st));   // self loops are never oriented
        count_launch(), k_triangles<false><<<tg, 256, 0, st>>>(M, d_ooff.get(), d_otgt.get(), d_oeid.get(), d_osrc.get(),
                                               d_cnt.get(), d_own.get(), nullptr, nullptr, nullptr);
        DRESS_TRY(exclusive_scan_i32(d_cnt.get(), d_ioff_old.get(), E, d_scan_tmp.get(), st));
        DRESS_CUDA_TRY(counted_memcpy(&T, d_ioff_old.get() + E, sizeof(T), cudaMemcpyDeviceToHost, st));
        DRESS_CUDA_TRY(cudaStreamSynchronize(st));
        DRESS_TRY(d_pairs_old.alloc((size_t)(T > 0 ? T : 1), st));
        DRESS_TRY(d_cursor.alloc((size_t)E, st));
        count_launch(), k_cursor_init<<<eg, 256, 0, st>>>(E, d_ioff_old.get(), d_own.get(), d_cursor.get());
        // The fill runs on the side stream, beside the edge validation, the
        // bins and the edge renumbering, which need only the counts; the main
        // stream joins it before the first read of the pairs (k_new_pairs).
        DRESS_CUDA_TRY(cudaEventRecord(ctx.fork, st));
        DRESS_CUDA_TRY(cudaStreamWaitEvent(ctx.side, ctx.fork, 0));
        fill.pending = true;
        count_launch(), k_triangles<true><<<tg, 256, 0, ctx.side>>>(M, d_ooff.get(), d_otgt.get(), d_oeid.get(),
                                                                    d_osrc.get(), nullptr, nullptr, d_ioff_old.get(),
                                                                    d_cursor.get(), d_pairs_old.get());
    } else {
        count_launch(), k_merge_intercepts<false><<<eg, 256, 0, st>>>(E, d_U.get(), d_V.get(), d_off.get(), d_tgt.get(),
                                                       d_eidx.get(), d_cnt.get(), nullptr, nullptr);
        DRESS_TRY(exclusive_scan_i32(d_cnt.get(), d_ioff_old.get(), E, d_scan_tmp.get(), st));
        DRESS_CUDA_TRY(counted_memcpy(&T, d_ioff_old.get() + E, sizeof(T), cudaMemcpyDeviceToHost, st));
        DRESS_CUDA_TRY(cudaStreamSynchronize(st));
        DRESS_TRY(d_pairs_old.alloc((size_t)(T > 0 ? T : 1), st));
        count_launch(), k_merge_intercepts<true><<<eg, 256, 0, st>>>(E, d_U.get(), d_V.get(), d_off.get(), d_tgt.get(),
                                                      d_eidx.get(), nullptr, d_ioff_old.get(),
                                                      d_pairs_old.get());
    }
    DRESS_CUDA_TRY(cudaGetLastError());
    if (tri_path) DRESS_TRY(validate_edges());
    d_tgt.release();

    // ---- bins and renumbering ---------------------------------------------------
    DevBuf<int> d_bc, d_vperm, d_vinv, d_eperm, d_einv;
    DRESS_TRY(d_bc.alloc(4 * NF, st));
    DRESS_TRY(d_vperm.alloc((size_t)N, st));
    DRESS_TRY(d_vinv.alloc((size_t)N, st));
    DRESS_TRY(d_eperm.alloc((size_t)E, st));
    DRESS_TRY(d_einv.alloc((size_t)E, st));
    DRESS_CUDA_TRY(cudaMemsetAsync(d_bc.get(), 0, 4 * NF * sizeof(int), st));
    const int vg = (int)grid_for(N, 256, 32 * sms);
    count_launch(), k_bin_count<<<vg, 256, 0, st>>>(N, d_deg.get(), d_bc.get());
    count_launch(), k_bin_count<<<eg, 256, 0, st>>>(E, d_cnt.get(), d_bc.get() + NF);
    DevBuf<unsigned long long> d_bterms;
    DRESS_TRY(d_bterms.alloc(2 * NB, st));
    DRESS_CUDA_TRY(cudaMemsetAsync(d_bterms.get(), 0, 2 * NB * sizeof(unsigned long long), st));
    count_launch(), k_bin_terms<<<vg, 256, 0, st>>>(N, d_deg.get(), d_bterms.get());
    count_launch(), k_bin_terms<<<eg, 256, 0, st>>>(E, d_cnt.get(), d_bterms.get() + NB);
    unsigned long long bterms[2 * NB];
    DRESS_CUDA_TRY(counted_memcpy(bterms, d_bterms.get(), sizeof(bterms), cudaMemcpyDeviceToHost, st));
    std::vector<int> bc(2 * NF);
    DRESS_CUDA_TRY(counted_memcpy(bc.data(), d_bc.get(), 2 * NF * sizeof(int), cudaMemcpyDeviceToHost, st));
    DRESS_CUDA_TRY(counted_memcpy(flags, d_flags.get(), sizeof(flags), cudaMemcpyDeviceToHost, st));
    DRESS_CUDA_TRY(cudaStreamSynchronize(st));
    const double t_pairs = ms_since(t0);
    if (flags[0]) return Status::Err(DRESSX_EINVAL, "malformed intercept tables");
    // fine ranges (cursors), then the coarse bins they make up
    std::vector<int> cur(2 * NF);
    cur[0] = 0;
    cur[NF] = 0;
    for (int f = 1; f < NF; ++f) {
        cur[f] = cur[f - 1] + bc[f - 1];
        cur[NF + f] = cur[NF + f - 1] + bc[NF + f - 1];
    }
    Bins vb, eb;
    for (int b = 0; b < NB; ++b) {
        vb.start[b] = cur[fine_first(b)];
        eb.start[b] = cur[NF + fine_first(b)];
    }
    vb.start[NB] = N;
    eb.start[NB] = E;
    // the warp bin, longest first, split where items have at most 256 and 64 terms
    for (int side = 0; side < 2; ++side) {
        Bins &bb = side ? eb : vb;
        const int base = side ? NF : 0;
        bb.med[0] = bb.start[BMED];
        bb.med[1] = cur[base + fine_of(256)];
        bb.med[2] = cur[base + fine_of(64)];
        bb.med[3] = bb.start[BMED + 1];
    }
    DRESS_CUDA_TRY(counted_memcpy(d_bc.get() + 2 * NF, cur.data(), 2 * NF * sizeof(int), cudaMemcpyHostToDevice, st));
    count_launch(), k_bin_scatter<<<vg, 256, 0, st>>>(N, d_deg.get(), d_bc.get() + 2 * NF, d_vperm.get(), d_vinv.get());
    // Edges of a large graph: one stable radix sort on (any pairs, owner,
    // other endpoint), for the locality of the sweeps' gathers.  A small
    // graph's sweeps are bound by launch latency and its arrays sit in L2, so
    // it keeps the one-pass scatter (the sort's passes cost more than they save).
    const bool locality = E >= LOCALITY_MIN_EDGES;
    if (!locality)
        count_launch(), k_bin_scatter<<<eg, 256, 0, st>>>(E, d_cnt.get(), d_bc.get() + 3 * NF, d_eperm.get(), d_einv.get());
    if (locality) {
        DevBuf<unsigned long long> k0, k1;
        DevBuf<unsigned> v0, v1;
        DRESS_TRY(k0.alloc((size_t)E, st));
        DRESS_TRY(k1.alloc((size_t)E, st));
        DRESS_TRY(v0.alloc((size_t)E, st));
        DRESS_TRY(v1.alloc((size_t)E, st));
        int vbits = 1;
        while (vbits < 31 && (1LL << vbits) < (long long)N) ++vbits;
        count_launch(), k_edge_keys<<<eg, 256, 0, st>>>(E, d_U.get(), d_V.get(), d_deg.get(), d_vinv.get(),
                                                        d_cnt.get(), vbits, k0.get(), v0.get());
        unsigned long long *sk = nullptr;
        unsigned *sv = nullptr;
        DRESS_TRY(sort_pairs(k0.get(), k1.get(), v0.get(), v1.get(), E, &sk, &sv, st, sms, 2 * vbits + 1));
        count_launch(), k_inverse<<<eg, 256, 0, st>>>(E, sv, d_eperm.get(), d_einv.get());
    }
    // block items largest first, so the longest sums start first (the sort
    // above already ordered the edges of a large graph)
    {
        struct Seg { int *perm, *inv; const int *len; int b0, b1; };
        Seg segs[4] = {{d_vperm.get(), d_vinv.get(), d_deg.get(), vb.start[BBLOCK], vb.start[BBLOCK + 1]},
                       {d_vperm.get(), d_vinv.get(), d_deg.get(), vb.start[BBIG], vb.start[BBIG + 1]},
                       {d_eperm.get(), d_einv.get(), d_cnt.get(), locality ? 0 : eb.start[BBLOCK], locality ? 0 : eb.start[BBLOCK + 1]},
                       {d_eperm.get(), d_einv.get(), d_cnt.get(), locality ? 0 : eb.start[BBIG], locality ? 0 : eb.start[BBIG + 1]}};
        for (const Seg &g2 : segs) {
            const int n = g2.b1 - g2.b0;
            if (n < 2) continue;
            DevBuf<int> d_len;
            DRESS_TRY(d_len.alloc((size_t)n, st));
            count_launch(), k_gather_seg<<<grid_for(n, 256, 64 * sms), 256, 0, st>>>(n, g2.perm + g2.b0, g2.len, d_len.get());
            std::vector<int> perm((size_t)n), len((size_t)n), idx((size_t)n);
            DRESS_CUDA_TRY(counted_memcpy(perm.data(), g2.perm + g2.b0, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost, st));
            DRESS_CUDA_TRY(counted_memcpy(len.data(), d_len.get(), (size_t)n * sizeof(int), cudaMemcpyDeviceToHost, st));
            DRESS_CUDA_TRY(cudaStreamSynchronize(st));
            for (int i = 0; i < n; ++i) idx[(size_t)i] = i;
            std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return len[(size_t)a] > len[(size_t)b]; });
            std::vector<int> sorted((size_t)n);
            for (int i = 0; i < n; ++i) sorted[(size_t)i] = perm[(size_t)idx[(size_t)i]];
            DRESS_CUDA_TRY(counted_memcpy(g2.perm + g2.b0, sorted.data(), (size_t)n * sizeof(int), cudaMemcpyHostToDevice, st));
            count_launch(), k_fix_inv<<<grid_for(n, 256, 64 * sms), 256, 0, st>>>(n, g2.b0, g2.perm, g2.inv);
            DRESS_CUDA_TRY(cudaStreamSynchronize(st));
        }
    }

    DevBuf<int> d_ndeg, d_row_eid, d_eu, d_ev, d_ncnt;
    DevBuf<long long> d_row_off, d_ioff;
    DevBuf<double> d_nwi, d_wi, d_dbuf, d_pbuf, d_vd;
    DevBuf<int2> d_pairs;
    DRESS_TRY(d_ndeg.alloc((size_t)N, st));
    DRESS_TRY(d_row_off.alloc((size_t)N + 1, st));
    DRESS_TRY(d_row_eid.alloc((size_t)(S > 0 ? S : 1), st));
    DRESS_TRY(d_nwi.alloc((size_t)N, st));
    count_launch(), k_gather_deg<<<vg, 256, 0, st>>>(N, d_vperm.get(), d_deg.get(), d_ndeg.get());
    DRESS_TRY(exclusive_scan_i32(d_ndeg.get(), d_row_off.get(), N, d_scan_tmp.get(), st));
    count_launch(), k_new_rows<<<grid_for((long long)N * 32, 256, 64 * sms), 256, 0, st>>>(
        N, d_vperm.get(), d_off.get(), d_eidx.get(), d_einv.get(), d_row_off.get(), d_row_eid.get(),
        d_nw.get(), d_nwi.get());
    if (locality) {                          // rows in edge-id order (vertex bins: thread, warp, block)
        const int t0 = vb.start[B2], t1 = vb.start[BMED], w1 = vb.start[BBLOCK], b1 = vb.start[BBIG];
        if (t1 > t0)
            count_launch(), k_sort_rows_thr<<<grid_for(t1 - t0, 256, 64 * sms), 256, 0, st>>>(t0, t1, d_row_off.get(),
                                                                                          d_row_eid.get());
        if (w1 > t1)
            count_launch(), k_sort_rows_warp<<<grid_for((long long)(w1 - t1) * 32, 32 * SORT_WARPS, 32 * sms),
                                               32 * SORT_WARPS, 0, st>>>(t1, w1, d_row_off.get(), d_row_eid.get());
        if (b1 > w1)
            count_launch(), k_sort_rows_blk<<<(unsigned)std::min(b1 - w1, 8 * sms), SORT_BLK_THR, 0, st>>>(
                w1, b1, d_row_off.get(), d_row_eid.get());
    }
    d_eidx.release();
    d_ndeg.release();

    DRESS_TRY(d_eu.alloc((size_t)E, st));
    DRESS_TRY(d_ev.alloc((size_t)E, st));
    DRESS_TRY(d_ncnt.alloc((size_t)E, st));
    DRESS_TRY(d_dbuf.alloc(2 * (size_t)E, st));
    if (!uniform) {
        DRESS_TRY(d_wi.alloc((size_t)E, st));
        DRESS_TRY(d_pbuf.alloc(2 * (size_t)E, st));
    }
    count_launch(), k_new_edges<<<eg, 256, 0, st>>>(E, d_eperm.get(), d_U.get(), d_V.get(), d_vinv.get(), d_w.get(),
                                    d_d.get(), d_cnt.get(), d_eu.get(), d_ev.get(),
                                    uniform ? nullptr : d_wi.get(), d_dbuf.get(),
                                    uniform ? nullptr : d_pbuf.get(), d_ncnt.get());
    DRESS_TRY(d_ioff.alloc((size_t)E + 1, st));
    DRESS_TRY(exclusive_scan_i32(d_ncnt.get(), d_ioff.get(), E, d_scan_tmp.get(), st));
    // The edges with common neighbours listed by size class (EdgeClasses):
    // a large graph sorts their ids by class; a small one's bins are already
    // in class order, so its list is their ids in order.
    EdgeClasses ec{};
    DevBuf<int> d_elist;
    const int e0 = eb.count(B0);
    ec.e0 = e0;
    DRESS_TRY(d_elist.alloc((size_t)std::max(1, E - e0), st));
    if (E - e0 > 0) {
        if (locality) {
            const int m = E - e0;
            DevBuf<unsigned long long> k0, k1;
            DevBuf<unsigned> v0, v1;
            DevBuf<int> d_bounds;
            DRESS_TRY(k0.alloc((size_t)m, st));
            DRESS_TRY(k1.alloc((size_t)m, st));
            DRESS_TRY(v0.alloc((size_t)m, st));
            DRESS_TRY(v1.alloc((size_t)m, st));
            DRESS_TRY(d_bounds.alloc(7, st));
            count_launch(), k_class_keys<<<grid_for(m, 256, 32 * sms), 256, 0, st>>>(e0, E, d_ncnt.get(), k0.get(),
                                                                                    v0.get());
            unsigned long long *sk = nullptr;
            unsigned *sv = nullptr;
            DRESS_TRY(sort_pairs(k0.get(), k1.get(), v0.get(), v1.get(), m, &sk, &sv, st, sms, 3));
            count_launch(), k_class_bounds<<<1, 32, 0, st>>>(m, sk, d_bounds.get());
            DRESS_CUDA_TRY(cudaMemcpyAsync(d_elist.get(), sv, (size_t)m * sizeof(int), cudaMemcpyDeviceToDevice, st));
            DRESS_CUDA_TRY(counted_memcpy(ec.cls, d_bounds.get(), 7 * sizeof(int), cudaMemcpyDeviceToHost, st));
            DRESS_CUDA_TRY(cudaStreamSynchronize(st));
            ec.cls[6] = m;
        } else {
            count_launch(), k_iota<<<grid_for(E - e0, 256, 32 * sms), 256, 0, st>>>(E - e0, e0, d_elist.get());
            const int b0 = e0;
            ec.cls[0] = eb.start[B2] - b0;
            ec.cls[1] = eb.start[BMED] - b0;
            ec.cls[2] = eb.med[1] - b0;
            ec.cls[3] = eb.med[2] - b0;
            ec.cls[4] = eb.med[3] - b0;
            ec.cls[5] = eb.start[BBIG] - b0;
            ec.cls[6] = E - b0;
        }
    }
    ec.list = d_elist.get();
    DRESS_TRY(d_pairs.alloc((size_t)(T > 0 ? T : 1), st));
    if (fill.pending) {                      // the pairs of the triangle listing are complete
        DRESS_CUDA_TRY(cudaEventRecord(ctx.join, ctx.side));
        DRESS_CUDA_TRY(cudaStreamWaitEvent(st, ctx.join, 0));
        fill.pending = false;
        d_otgt.release(); d_oeid.release(); d_osrc.release(); d_ooff.release(); d_ocnt.release();
        d_cursor.release(); d_own.release();
    }
    if (E - e0 > 0) {
        const int c1 = ec.cls[1], c6 = ec.cls[6];
        if (c1 > 0)
            count_launch(), k_new_pairs<1><<<grid_for(c1, 256, 64 * sms), 256, 0, st>>>(
                ec.list, 0, c1, d_eperm.get(), d_ioff_old.get(), d_pairs_old.get(), d_einv.get(), d_ioff.get(),
                d_pairs.get());
        if (c6 > c1)
            count_launch(), k_new_pairs<32><<<grid_for((long long)(c6 - c1) * 32, 256, 64 * sms), 256, 0, st>>>(
                ec.list, c1, c6, d_eperm.get(), d_ioff_old.get(), d_pairs_old.get(), d_einv.get(), d_ioff.get(),
                d_pairs.get());
    }
    DRESS_CUDA_TRY(cudaGetLastError());
    d_pairs_old.release();
    // each edge's pairs in edge-id order (class lists: thread, warp and block sorts)
    if (locality && T > 1) {
        const int *L = ec.list;
        const int c0 = ec.cls[0], c1 = ec.cls[1], c4 = ec.cls[4], c5 = ec.cls[5];
        if (c1 > c0)
            count_launch(), k_sort_pairs_thr<<<grid_for(c1 - c0, 256, 64 * sms), 256, 0, st>>>(L, c0, c1, d_ioff.get(),
                                                                                             d_pairs.get());
        if (c4 > c1)
            count_launch(), k_sort_pairs_warp<<<grid_for((long long)(c4 - c1) * 32, 32 * SORT_WARPS, 32 * sms),
                                               32 * SORT_WARPS, 0, st>>>(L, c1, c4, d_ioff.get(), d_pairs.get());
        if (c5 > c4)
            count_launch(), k_sort_pairs_blk<<<(unsigned)std::min(c5 - c4, 8 * sms), SORT_BLK_THR, 0, st>>>(
                L, c4, c5, d_ioff.get(), d_pairs.get());
        DRESS_CUDA_TRY(cudaGetLastError());
    }
    d_U.release(); d_V.release(); d_w.release(); d_d.release(); d_nw.release();
    d_ioff_old.release(); d_ncnt.release(); d_cnt.release(); d_deg.release();

    // exact sums of queued items: shared memory for their terms, a global
    // scratch slice per block for items beyond it
    int smem_optin = 0;
    DRESS_CUDA_TRY(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx.device));
    const int exact_cap = (smem_optin - 2048) / 8;
    const long long max_terms = max_row + 1;       // a row's slots or an edge's pairs, plus the self term
    const int exact_grid = max_terms > exact_cap ? std::min(32, 2 * sms) : 2 * sms;
    DevBuf<double> d_scratch;
    long long scratch_stride = 0;
    if (max_terms > exact_cap) {
        scratch_stride = (max_terms + 31) & ~31LL;
        DRESS_TRY(d_scratch.alloc((size_t)exact_grid * (size_t)scratch_stride, st));
    }
    const size_t exact_smem = (size_t)exact_cap * sizeof(double);
    DRESS_TRY(set_sweep_attributes<true>(exact_smem));
    DRESS_TRY(set_sweep_attributes<false>(exact_smem));

    DevBuf<unsigned long long> d_maxd;
    DRESS_TRY(d_vd.alloc((size_t)(N > 0 ? N : 1), st));
    DRESS_TRY(d_maxd.alloc(RING, st));
    DRESS_CUDA_TRY(cudaStreamSynchronize(st));
    double setup_ms = ms_since(t0);
    cudaEvent_t sw0, sw1;
    DRESS_CUDA_TRY(cudaEventCreate(&sw0));
    DRESS_CUDA_TRY(cudaEventCreate(&sw1));
    DRESS_CUDA_TRY(cudaEventRecord(sw0, st));

    // ---- sweeps -------------------------------------------------------------
    Sweep s;
    s.N = N; s.E = E; s.fwd = fwd;
    s.row_off = d_row_off.get(); s.row_eid = d_row_eid.get();
    s.eu = d_eu.get(); s.ev = d_ev.get();
    s.w = uniform ? nullptr : d_wi.get();
    s.wc = wc;
    bool unit_nw = true;                       // NULL vertex weights mean all 1.0
    if (g->NW)
        for (int i = 0; i < N && unit_nw; ++i) unit_nw = g->NW[i] == 1.0;
    s.nw = unit_nw ? nullptr : d_nwi.get();
    s.ioff = d_ioff.get(); s.pairs = d_pairs.get();
    s.vd = d_vd.get(); s.maxd = d_maxd.get();
    s.eps = epsilon;
    s.scratch = d_scratch.get(); s.scratch_stride = scratch_stride; s.exact_cap = exact_cap;
    s.force_exact = ctx.cfg->exact_sums != 0;
    DevBuf<int> d_qv, d_qe;
    DevBuf<unsigned> d_qcount;
    DRESS_TRY(d_qv.alloc((size_t)(N > 0 ? N : 1), st));
    DRESS_TRY(d_qe.alloc((size_t)(E > 0 ? E : 1), st));
    DRESS_TRY(d_qcount.alloc(2, st));
    DRESS_CUDA_TRY(cudaMemsetAsync(d_qcount.get(), 0, 2 * sizeof(unsigned), st));
    s.qv = d_qv.get(); s.qe = d_qe.get(); s.qcount = d_qcount.get();
    LaunchCfg lc{sms, exact_grid, exact_smem, st, ctx.side, ctx.fork, ctx.join};
    double *dbuf[2] = {d_dbuf.get(), d_dbuf.get() + E};
    double *pbuf[2] = {uniform ? nullptr : d_pbuf.get(), uniform ? nullptr : d_pbuf.get() + E};

    // Two sweeps (the even one writes buffer 1, the odd one buffer 0) and the
    // index steps between them are captured once into a CUDA graph, replayed
    // for every pair of sweeps; the host reads the ring after each chunk.
    DevBuf<int> d_iter;
    DRESS_TRY(d_iter.alloc(1, st));
    DRESS_CUDA_TRY(cudaMemsetAsync(d_iter.get(), 0, sizeof(int), st));
    DRESS_CUDA_TRY(cudaMemsetAsync(d_maxd.get(), 0, RING * sizeof(unsigned long long), st));
    s.iter = d_iter.get();
    s.max_iter = max_iterations;
    Sweep sw2[2] = {s, s};
    for (int par = 0; par < 2; ++par) {
        sw2[par].d = dbuf[par]; sw2[par].dn = dbuf[par ^ 1];
        sw2[par].p = pbuf[par]; sw2[par].pn = pbuf[par ^ 1];
    }
    auto enqueue_pair = [&]() -> Status {
        for (int par = 0; par < 2; ++par) {
            if (uniform) DRESS_TRY(launch_sweep<true>(sw2[par], vb, ec, lc));
            else         DRESS_TRY(launch_sweep<false>(sw2[par], vb, ec, lc));
            count_launch(), k_next_sweep<<<1, 1, 0, st>>>(d_iter.get(), d_maxd.get());
            DRESS_CUDA_TRY(cudaGetLastError());
        }
        return Status::Ok();
    };
    cudaGraphExec_t gexec = nullptr;
    long long pair_launches = 0;
    {
        DRESS_CUDA_TRY(cudaStreamSynchronize(st));
        const long long before = tls_launches;
        cudaGraph_t graph = nullptr;
        if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
            Status cs = enqueue_pair();
            cudaError_t e = cudaStreamEndCapture(st, &graph);
            if (cs.ok() && e == cudaSuccess && graph && cudaGraphInstantiate(&gexec, graph, 0) != cudaSuccess)
                gexec = nullptr;
            if (graph) cudaGraphDestroy(graph);
        }
        cudaGetLastError();                           // a failed capture leaves direct launches
        pair_launches = tls_launches - before;
        engine().launches -= pair_launches;           // counted per replay below
        tls_launches -= pair_launches;
    }
    struct GraphGuard {
        cudaGraphExec_t g;
        ~GraphGuard() { if (g) cudaGraphExecDestroy(g); }
    } guard{gexec};
    unsigned long long hmax[RING];
    int conv = -1, done = 0;
    int chunk = ctx.cfg->fit_chunk > 0 ? (ctx.cfg->fit_chunk < MAX_CHUNK ? ctx.cfg->fit_chunk : MAX_CHUNK) : 8;
    chunk = (chunk + 1) & ~1;
    double last_delta = 0.0;
    while (done < max_iterations && conv < 0) {
        for (int r = 0; r < chunk / 2; ++r) {
            if (gexec) {
                count_launch((int)pair_launches);
                DRESS_CUDA_TRY(cudaGraphLaunch(gexec, st));
            } else {
                DRESS_TRY(enqueue_pair());
            }
        }
        const int hi = done + chunk < max_iterations ? done + chunk : max_iterations;
        DRESS_CUDA_TRY(counted_memcpy(hmax, d_maxd.get(), RING * sizeof(unsigned long long),
                                       cudaMemcpyDeviceToHost, st));
        DRESS_CUDA_TRY(cudaStreamSynchronize(st));
        for (int it = done; it < hi; ++it) {
            double m;
            std::memcpy(&m, &hmax[it % RING], sizeof(m));
            last_delta = m;
            if (m < epsilon) { conv = it; break; }
        }
        done = hi;
        // Next chunk: the sweeps that the decay of the last three deltas
        // predicts until the tolerance, plus two, when they decay; else twice
        // the last chunk.  Sweeps past convergence return at once but still
        // cost their launches (≈ 3 µs each), a short chunk costs one more
        // host round trip.
        int next = chunk < MAX_CHUNK ? 2 * chunk : MAX_CHUNK;
        if (conv < 0 && done >= 4) {
            double m1, m0;
            std::memcpy(&m1, &hmax[(done - 1) % RING], sizeof(m1));
            std::memcpy(&m0, &hmax[(done - 4) % RING], sizeof(m0));
            if (m1 >= epsilon && m1 > 0.0 && m0 > m1) {
                const double rate = std::pow(m1 / m0, 1.0 / 3.0);
                const double need = std::log(epsilon / m1) / std::log(rate);
                if (need >= 0.0 && need < (double)MAX_CHUNK) next = std::max(2, (int)std::ceil(need) + 2);
            }
        }
        chunk = std::min(MAX_CHUNK, (next + 1) & ~1);
    }
    const int last = conv >= 0 ? conv : max_iterations - 1;
    // device time of the sweeps (the chunk tails after convergence return at once)
    DRESS_CUDA_TRY(cudaEventRecord(sw1, st));
    DRESS_CUDA_TRY(cudaEventSynchronize(sw1));
    float sweep_ms = 0.f;
    cudaEventElapsedTime(&sweep_ms, sw0, sw1);
    cudaEventDestroy(sw0);
    cudaEventDestroy(sw1);

    // ---- results back in the caller's numbering ------------------------------
    DevBuf<double> d_out;
    DRESS_TRY(d_out.alloc((size_t)E + N + 1, st));
    const auto t_down0 = std::chrono::steady_clock::now();
    count_launch(), k_unpermute<<<eg, 256, 0, st>>>(E, d_eperm.get(), dbuf[(last + 1) & 1], d_out.get());
    count_launch(), k_unpermute<<<vg, 256, 0, st>>>(N, d_vperm.get(), d_vd.get(), d_out.get() + E);
    {
        const HostSpan spans[2] = {{g->edge_dress, d_out.get(), (size_t)E * sizeof(double)},
                                   {g->vertex_dress, d_out.get() + E, (size_t)N * sizeof(double)}};
        DRESS_TRY(staged_download(spans, 2, ctx));
    }
    if (iterations) *iterations = conv >= 0 ? conv : max_iterations;
    if (delta) *delta = last_delta;
    if (stats) {
        for (int b = 0; b < NB && b < 8; ++b) {
            stats->vbin_items[b] = vb.count(b);
            stats->ebin_items[b] = eb.count(b);
            stats->vbin_terms[b] = (long long)bterms[b];
            stats->ebin_terms[b] = (long long)bterms[NB + b];
        }
        stats->T = T;
        stats->sweeps = last + 1;
        stats->setup_ms = setup_ms;
        stats->iterate_ms = sweep_ms;
        stats->phase_ms[0] = t_upload + edge_up.wait_ms;
        stats->phase_ms[1] = t_valid;
        stats->phase_ms[2] = t_pairs - t_upload - edge_up.wait_ms - t_valid;
        stats->phase_ms[3] = setup_ms - t_pairs;
        stats->phase_ms[4] = ms_since(t_down0);
    }
    return Status::Ok();
}

}  // namespace dress
