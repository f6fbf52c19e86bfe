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
#include <climits>
#include <chrono>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "engine.h"

namespace dress {
namespace {

constexpr int NB = 8;
constexpr int RING = 64;           // per-sweep convergence slots
constexpr int MAX_CHUNK = 32;      // sweeps launched per host check (<= RING/2)
constexpr int WARP_CAP = 1024;     // terms one warp sorts in shared memory
enum { B1 = 0, B2, B4, B8, B16, B32, BWARP, BBLOCK };

__host__ __device__ __forceinline__ int bin_of(long long n)
{
    return n <= 1 ? B1 : n <= 2 ? B2 : n <= 4 ? B4 : n <= 8 ? B8 : n <= 16 ? B16
         : n <= 32 ? B32 : n <= WARP_CAP ? BWARP : BBLOCK;
}

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
__global__ void k_validate_rows(int N, int E, const int *off, const int *tgt, const int *eidx,
                                int *deg, int *flags)
{
    for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < N; u += gridDim.x * blockDim.x) {
        int b = off[u], e = off[u + 1];
        if (e < b) { atomicOr(&flags[0], 1); deg[u] = 0; continue; }
        deg[u] = e - b;
        atomicMax(&flags[3], e - b);
        int prev = -1;
        for (int s = b; s < e; ++s) {
            int x = tgt[s], ei = eidx[s];
            if (x < 0 || x >= N || ei < 0 || ei >= E) { atomicOr(&flags[0], 2); break; }
            if (s > b) {
                if (x == prev) flags[1] = 1;
                else if (x < prev) atomicOr(&flags[0], 4);
            }
            prev = x;
        }
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

__global__ void k_orient_count(int N, const int *off, const int *tgt, const int *deg, int *ocnt)
{
    for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < N; u += gridDim.x * blockDim.x) {
        unsigned long long ku = rank_key(deg, u);
        int c = 0;
        for (int s = off[u]; s < off[u + 1]; ++s) c += rank_key(deg, tgt[s]) > ku;
        ocnt[u] = c;
    }
}

__global__ void k_orient_fill(int N, const int *off, const int *tgt, const int *eidx, const int *deg,
                              const long long *ooff, int *otgt, int *oeid, int *osrc)
{
    for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < N; u += gridDim.x * blockDim.x) {
        unsigned long long ku = rank_key(deg, u);
        long long q = ooff[u];
        for (int s = off[u]; s < off[u + 1]; ++s) {
            int x = tgt[s];
            if (rank_key(deg, x) > ku) { otgt[q] = x; oeid[q] = eidx[s]; osrc[q] = u; ++q; }
        }
    }
}

// Each oriented edge a->b intersects out(a) with out(b) (both ascending by id).
// A common c closes the triangle {a,b,c}; each of its three edges receives
// the pair of the other two (the order inside a pair is irrelevant: the term
// is their sum).
template <bool FILL>
__global__ void k_triangles(long long M, const long long *ooff, const int *otgt, const int *oeid,
                            const int *osrc, int *cnt, unsigned long long *cursor, int2 *pairs)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < M;
         q += (long long)gridDim.x * blockDim.x) {
        int a = osrc[q], b = otgt[q], eab = oeid[q];
        long long pa = ooff[a], pa_end = ooff[a + 1];
        long long pb = ooff[b], pb_end = ooff[b + 1];
        while (pa < pa_end && pb < pb_end) {
            int x = otgt[pa], y = otgt[pb];
            if (x == y) {
                int eac = oeid[pa], ebc = oeid[pb];
                if (!FILL) {
                    atomicAdd(&cnt[eab], 1);
                    atomicAdd(&cnt[eac], 1);
                    atomicAdd(&cnt[ebc], 1);
                } else {
                    pairs[atomicAdd(&cursor[eab], 1ULL)] = make_int2(eac, ebc);
                    pairs[atomicAdd(&cursor[eac], 1ULL)] = make_int2(eab, ebc);
                    pairs[atomicAdd(&cursor[ebc], 1ULL)] = make_int2(eab, eac);
                }
                ++pa;
                ++pb;
            } else if (x < y) {
                ++pa;
            } else {
                ++pb;
            }
        }
    }
}

__global__ void k_copy_i64(long long n, const long long *src, unsigned long long *dst)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        dst[i] = (unsigned long long)src[i];
}

// ---- binning (terms per item) and renumbering ----
__global__ void k_bin_count(int n, const int *len, int add, int *bin_cnt)
{
    __shared__ int sc[NB];
    if (threadIdx.x < NB) sc[threadIdx.x] = 0;
    __syncthreads();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        atomicAdd(&sc[bin_of((long long)len[i] + add)], 1);
    __syncthreads();
    if (threadIdx.x < NB && sc[threadIdx.x]) atomicAdd(&bin_cnt[threadIdx.x], sc[threadIdx.x]);
}

// Scatter items into their bins; lanes of a warp that share a bin take
// consecutive slots (one atomic per group), which keeps neighbouring items
// neighbours.
__global__ void k_bin_scatter(int n, const int *len, int add, int *cursor, int *perm, int *inv)
{
    int lane = threadIdx.x & 31;
    for (int i0 = blockIdx.x * blockDim.x; i0 < n; i0 += gridDim.x * blockDim.x) {
        int i = i0 + threadIdx.x;
        unsigned active = __ballot_sync(0xffffffffu, i < n);
        if (i < n) {
            int b = bin_of((long long)len[i] + add);
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

__global__ void k_new_pairs(int E, const int *eperm, const long long *ioff_old, const int2 *pairs_old,
                            const int *einv, const long long *ioff_new, int2 *pairs_new)
{
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < E; j += gridDim.x * blockDim.x) {
        int e = eperm[j];
        long long a = ioff_old[e], n = ioff_old[e + 1] - a, o = ioff_new[j];
        for (long long k = 0; k < n; ++k) {
            int2 pr = pairs_old[a + k];
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

// ------------------------------------------------------------------------
// sweep kernels
// ------------------------------------------------------------------------

struct Sweep {
    int N, E, fwd;                 // fwd: FORWARD/BACKWARD self term
    const long long *row_off;      // [N+1] renumbered CSR rows
    const int *row_eid;            // [S]
    const int *eu, *ev;            // [E]
    const double *w;               // [E] (weighted graphs)
    double wc;                     // the weight when all are equal
    const double *nw;              // [N]
    const long long *ioff;         // [E+1]
    const int2 *pairs;             // [T]
    double *vd;                    // [N]
    unsigned long long *maxd;      // [max_iterations]
    const double *d, *p;           // current values and products
    double *dn, *pn;               // next values and products
    int iter, slot, prev_slot;     // sweep index and its convergence slots
    double eps;
    double *scratch;               // block-bin spill area (rows larger than shared memory)
    long long scratch_stride;
};

template <bool UNIF>
__device__ __forceinline__ double prod(const Sweep &s, int e)
{
    return UNIF ? dmul(s.wc, s.d[e]) : s.p[e];
}

template <bool UNIF>
__device__ __forceinline__ double self_term(const Sweep &s, int j, int u, int v)
{
    double own = prod<UNIF>(s, j);
    double a = dmul(4.0, s.nw[u]);
    if (s.fwd) return dadd(a, own);
    return dadd(dadd(a, dmul(4.0, s.nw[v])), dmul(2.0, own));
}

// edge value from its sorted-KBN numerator; also stores d_next (and p_next)
template <bool UNIF>
__device__ __forceinline__ double finish_edge(const Sweep &s, int j, int u, int v, double num)
{
    double den = dmul(s.vd[u], s.vd[v]);
    double r = den > 0.0 ? ddiv(num, den) : 0.0;
    s.dn[j] = r;
    if (!UNIF) s.pn[j] = dmul(s.w[j], r);
    return fabs(dsub(s.d[j], r));
}

// ---- one thread per item, M-term register network ----
template <int M, bool UNIF>
__global__ void __launch_bounds__(128) k_vertex_thr(Sweep s, int begin, int end)
{
    if (s.iter > 0 && __longlong_as_double((long long)s.maxd[s.prev_slot]) < s.eps) return;
    int i = begin + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= end) return;
    long long b = s.row_off[i];
    int deg = (int)(s.row_off[i + 1] - b);
    double a[M];
    a[0] = dmul(4.0, s.nw[i]);
#pragma unroll
    for (int k = 1; k < M; ++k) a[k] = (k <= deg) ? prod<UNIF>(s, s.row_eid[b + k - 1]) : DRESS_INF;
    if (M > 1) sort_regs<M>(a);
    s.vd[i] = dsqrt(kbn_regs<M>(a, deg + 1));
}

template <int M, bool UNIF>
__global__ void __launch_bounds__(128) k_edge_thr(Sweep s, int begin, int end)
{
    if (s.iter > 0 && __longlong_as_double((long long)s.maxd[s.prev_slot]) < s.eps) return;
    int j = begin + blockIdx.x * blockDim.x + threadIdx.x;
    double delta = 0.0;
    if (j < end) {
        int u = s.eu[j], v = s.ev[j];
        double self = self_term<UNIF>(s, j, u, v);
        double num;
        if (M == 1) {
            num = dadd(self, 0.0);           // sorted KBN of a single term
        } else {
            long long o = s.ioff[j];
            int nc = (int)(s.ioff[j + 1] - o);
            double a[M];
#pragma unroll
            for (int k = 0; k < M; ++k) {
                if (k < nc) {
                    int2 pr = s.pairs[o + k];
                    a[k] = dadd(prod<UNIF>(s, pr.x), prod<UNIF>(s, pr.y));
                } else {
                    a[k] = (k == nc) ? self : DRESS_INF;
                }
            }
            sort_regs<M>(a);
            num = kbn_regs<M>(a, nc + 1);
        }
        delta = finish_edge<UNIF>(s, j, u, v, num);
    }
    block_max_to(&s.maxd[s.slot], delta);
}

// ---- one warp per item, shared-memory sort ----
struct WarpSync { __device__ void operator()() const { __syncwarp(); } };
struct BlockSync { __device__ void operator()() const { __syncthreads(); } };

template <bool UNIF>
__global__ void __launch_bounds__(256) k_vertex_warp(Sweep s, int begin, int end)
{
    extern __shared__ double sm[];
    if (s.iter > 0 && __longlong_as_double((long long)s.maxd[s.prev_slot]) < s.eps) return;
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    double *buf = sm + (size_t)wid * WARP_CAP;
    for (int i = begin + blockIdx.x * nw + wid; i < end; i += gridDim.x * nw) {
        long long b = s.row_off[i];
        int deg = (int)(s.row_off[i + 1] - b), n = deg + 1;
        if (lane == 0) buf[0] = dmul(4.0, s.nw[i]);
        for (int k = lane; k < deg; k += 32) buf[k + 1] = prod<UNIF>(s, s.row_eid[b + k]);
        __syncwarp();
        sort_shared(buf, n, lane, 32, WarpSync());
        if (lane == 0) s.vd[i] = dsqrt(kbn_sorted_buf(buf, n));
        __syncwarp();
    }
}

template <bool UNIF>
__global__ void __launch_bounds__(256) k_edge_warp(Sweep s, int begin, int end)
{
    extern __shared__ double sm[];
    if (s.iter > 0 && __longlong_as_double((long long)s.maxd[s.prev_slot]) < s.eps) return;
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    double *buf = sm + (size_t)wid * WARP_CAP;
    double delta = 0.0;
    for (int j = begin + blockIdx.x * nw + wid; j < end; j += gridDim.x * nw) {
        int u = s.eu[j], v = s.ev[j];
        long long o = s.ioff[j];
        int nc = (int)(s.ioff[j + 1] - o);
        for (int k = lane; k < nc; k += 32) {
            int2 pr = s.pairs[o + k];
            buf[k] = dadd(prod<UNIF>(s, pr.x), prod<UNIF>(s, pr.y));
        }
        if (lane == 0) buf[nc] = self_term<UNIF>(s, j, u, v);
        __syncwarp();
        sort_shared(buf, nc + 1, lane, 32, WarpSync());
        if (lane == 0) delta = fmax(delta, finish_edge<UNIF>(s, j, u, v, kbn_sorted_buf(buf, nc + 1)));
        __syncwarp();
    }
    block_max_to(&s.maxd[s.slot], delta);
}

// ---- one block per item (hub rows / hub edges) ----
template <bool UNIF>
__global__ void __launch_bounds__(512) k_vertex_block(Sweep s, int begin, int end, int cap)
{
    extern __shared__ double sm[];
    if (s.iter > 0 && __longlong_as_double((long long)s.maxd[s.prev_slot]) < s.eps) return;
    for (int i = begin + blockIdx.x; i < end; i += gridDim.x) {
        long long b = s.row_off[i];
        int deg = (int)(s.row_off[i + 1] - b), n = deg + 1;
        double *buf = n <= cap ? sm : s.scratch + (long long)blockIdx.x * s.scratch_stride;
        if (threadIdx.x == 0) buf[0] = dmul(4.0, s.nw[i]);
        for (int k = threadIdx.x; k < deg; k += blockDim.x) buf[k + 1] = prod<UNIF>(s, s.row_eid[b + k]);
        __syncthreads();
        sort_shared(buf, n, threadIdx.x, blockDim.x, BlockSync());
        if (threadIdx.x == 0) s.vd[i] = dsqrt(kbn_sorted_buf(buf, n));
        __syncthreads();
    }
}

template <bool UNIF>
__global__ void __launch_bounds__(512) k_edge_block(Sweep s, int begin, int end, int cap)
{
    extern __shared__ double sm[];
    if (s.iter > 0 && __longlong_as_double((long long)s.maxd[s.prev_slot]) < s.eps) return;
    double delta = 0.0;
    for (int j = begin + blockIdx.x; j < end; j += gridDim.x) {
        int u = s.eu[j], v = s.ev[j];
        long long o = s.ioff[j];
        int nc = (int)(s.ioff[j + 1] - o);
        double *buf = nc + 1 <= cap ? sm : s.scratch + (long long)blockIdx.x * s.scratch_stride;
        for (int k = threadIdx.x; k < nc; k += blockDim.x) {
            int2 pr = s.pairs[o + k];
            buf[k] = dadd(prod<UNIF>(s, pr.x), prod<UNIF>(s, pr.y));
        }
        if (threadIdx.x == 0) buf[nc] = self_term<UNIF>(s, j, u, v);
        __syncthreads();
        sort_shared(buf, nc + 1, threadIdx.x, blockDim.x, BlockSync());
        if (threadIdx.x == 0) delta = fmax(delta, finish_edge<UNIF>(s, j, u, v, kbn_sorted_buf(buf, nc + 1)));
        __syncthreads();
    }
    block_max_to(&s.maxd[s.slot], delta);
}

// ------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------

inline unsigned grid_for(long long n, int threads, int cap_blocks)
{
    long long b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > cap_blocks) b = cap_blocks;
    return (unsigned)b;
}

struct Bins {
    int start[NB + 1];
    long long max_terms_block;   // largest item in the block bin
};

template <bool UNIF>
Status launch_sweep(const Sweep &s, const Bins &vb, const Bins &eb, int sms, int block_cap,
                    cudaStream_t st)
{
    const int T = 128;
    // hub items first: they carry the longest sequential sums
    if (vb.start[BBLOCK + 1] > vb.start[BBLOCK]) {
        int n = vb.start[BBLOCK + 1] - vb.start[BBLOCK];
        count_launch(), k_vertex_block<UNIF><<<grid_for(n, 1, 2 * sms), 512, (size_t)block_cap * 8, st>>>(
            s, vb.start[BBLOCK], vb.start[BBLOCK + 1], block_cap);
    }
    if (vb.start[BWARP + 1] > vb.start[BWARP]) {
        int n = vb.start[BWARP + 1] - vb.start[BWARP];
        count_launch(), k_vertex_warp<UNIF><<<grid_for(n, 8, 8 * sms), 256, 8 * WARP_CAP * 8, st>>>(
            s, vb.start[BWARP], vb.start[BWARP + 1]);
    }
#define DRESS_VTHR(BIN, M)                                                                   \
    if (vb.start[BIN + 1] > vb.start[BIN])                                                   \
        count_launch(), k_vertex_thr<M, UNIF><<<grid_for(vb.start[BIN + 1] - vb.start[BIN], T, INT_MAX), T, 0, st>>>( \
            s, vb.start[BIN], vb.start[BIN + 1]);
    DRESS_VTHR(B32, 32) DRESS_VTHR(B16, 16) DRESS_VTHR(B8, 8) DRESS_VTHR(B4, 4) DRESS_VTHR(B2, 2)
    DRESS_VTHR(B1, 1)
#undef DRESS_VTHR
    if (eb.start[BBLOCK + 1] > eb.start[BBLOCK]) {
        int n = eb.start[BBLOCK + 1] - eb.start[BBLOCK];
        count_launch(), k_edge_block<UNIF><<<grid_for(n, 1, 2 * sms), 512, (size_t)block_cap * 8, st>>>(
            s, eb.start[BBLOCK], eb.start[BBLOCK + 1], block_cap);
    }
    if (eb.start[BWARP + 1] > eb.start[BWARP]) {
        int n = eb.start[BWARP + 1] - eb.start[BWARP];
        count_launch(), k_edge_warp<UNIF><<<grid_for(n, 8, 8 * sms), 256, 8 * WARP_CAP * 8, st>>>(
            s, eb.start[BWARP], eb.start[BWARP + 1]);
    }
#define DRESS_ETHR(BIN, M)                                                                   \
    if (eb.start[BIN + 1] > eb.start[BIN])                                                   \
        count_launch(), k_edge_thr<M, UNIF><<<grid_for(eb.start[BIN + 1] - eb.start[BIN], T, INT_MAX), T, 0, st>>>( \
            s, eb.start[BIN], eb.start[BIN + 1]);
    DRESS_ETHR(B32, 32) DRESS_ETHR(B16, 16) DRESS_ETHR(B8, 8) DRESS_ETHR(B4, 4) DRESS_ETHR(B2, 2)
    DRESS_ETHR(B1, 1)
#undef DRESS_ETHR
    DRESS_CUDA_TRY(cudaGetLastError());
    return Status::Ok();
}

template <class T>
Status upload(DevBuf<T> &b, const T *host, size_t n, cudaStream_t st)
{
    DRESS_TRY(b.alloc(n, st));
    if (n) DRESS_CUDA_TRY(counted_memcpy(b.get(), host, n * sizeof(T), cudaMemcpyHostToDevice, st));
    return Status::Ok();
}

double ms_since(std::chrono::steady_clock::time_point t0)
{
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

Status fit_graph(p_dress_graph_t g, int max_iterations, double epsilon, int *iterations,
                 double *delta, FitStats *stats)
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

    Engine &en = engine();
    cudaStream_t st = en.stream;
    const int sms = en.num_sms;
    const int fwd = (g->variant == DRESS_VARIANT_FORWARD || g->variant == DRESS_VARIANT_BACKWARD);

    // ---- upload --------------------------------------------------------
    DevBuf<int> d_off, d_tgt, d_eidx, d_U, d_V;
    DevBuf<double> d_w, d_d, d_nw;
    DRESS_TRY(upload(d_off, g->adj_offset, (size_t)N + 1, st));
    DRESS_TRY(upload(d_tgt, g->adj_target, (size_t)S, st));
    DRESS_TRY(upload(d_eidx, g->adj_edge_idx, (size_t)S, st));
    DRESS_TRY(upload(d_U, g->U, (size_t)E, st));
    DRESS_TRY(upload(d_V, g->V, (size_t)E, st));
    DRESS_TRY(upload(d_w, g->edge_weight, (size_t)E, st));
    DRESS_TRY(upload(d_d, g->edge_dress, (size_t)E, st));
    if (g->NW) {
        DRESS_TRY(upload(d_nw, g->NW, (size_t)N, st));
    } else {                                   // NULL vertex weights mean all 1.0
        DRESS_TRY(d_nw.alloc((size_t)N, st));
        if (N) count_launch(), k_fill<<<grid_for(N, 256, 16 * sms), 256, 0, st>>>(N, 1.0, d_nw.get());
    }

    // ---- validate ----------------------------------------------------------
    DevBuf<int> d_flags, d_deg, d_cnt;
    DRESS_TRY(d_flags.alloc(8, st));
    DRESS_TRY(d_deg.alloc((size_t)N, st));
    DRESS_TRY(d_cnt.alloc((size_t)E, st));
    DRESS_CUDA_TRY(cudaMemsetAsync(d_flags.get(), 0, 8 * sizeof(int), st));
    count_launch(), k_validate_rows<<<grid_for(N, 256, 16 * sms), 256, 0, st>>>(N, E, d_off.get(), d_tgt.get(),
                                                                d_eidx.get(), d_deg.get(), d_flags.get());
    count_launch(), k_validate_edges<<<grid_for(E, 256, 16 * sms), 256, 0, st>>>(N, E, d_U.get(), d_V.get(), d_w.get(),
                                                                 d_flags.get());
    DRESS_CUDA_TRY(cudaGetLastError());
    int flags[8];
    DRESS_CUDA_TRY(counted_memcpy(flags, d_flags.get(), sizeof(flags), cudaMemcpyDeviceToHost, st));
    DRESS_CUDA_TRY(cudaStreamSynchronize(st));
    if (flags[0]) return Status::Err(DRESSX_EINVAL, "malformed graph (CSR or edge endpoints out of range)");
    const bool dup = flags[1] != 0;
    const bool uniform = flags[2] == 0;
    const double wc = E > 0 ? g->edge_weight[0] : 1.0;
    const long long max_row = flags[3];

    // ---- common-neighbour tables (original edge ids) -------------------------
    DevBuf<long long> d_ioff_old, d_scan_tmp;
    DevBuf<int2> d_pairs_old;
    DRESS_TRY(d_ioff_old.alloc((size_t)E + 1, st));
    DRESS_TRY(d_scan_tmp.alloc(scan_tmp_elems((long long)(S > E ? S : E) + N + 1), st));
    long long T = 0;
    const int eg = (int)grid_for(E, 256, 32 * sms);
    if (g->precompute_intercepts && g->intercept_offset) {
        DevBuf<int> d_io, d_ux, d_vx;
        DRESS_TRY(upload(d_io, g->intercept_offset, (size_t)E + 1, st));
        long long Tg = g->intercept_offset[E];
        if (Tg < 0) return Status::Err(DRESSX_EINVAL, "bad intercept_offset");
        DRESS_TRY(upload(d_ux, g->intercept_edge_ux, (size_t)Tg, st));
        DRESS_TRY(upload(d_vx, g->intercept_edge_vx, (size_t)Tg, st));
        count_launch(), k_given_counts<<<eg, 256, 0, st>>>(E, d_io.get(), d_cnt.get(), d_flags.get());
        DRESS_TRY(exclusive_scan_i32(d_cnt.get(), d_ioff_old.get(), E, d_scan_tmp.get(), st));
        DRESS_CUDA_TRY(counted_memcpy(&T, d_ioff_old.get() + E, sizeof(T), cudaMemcpyDeviceToHost, st));
        DRESS_CUDA_TRY(cudaStreamSynchronize(st));
        DRESS_TRY(d_pairs_old.alloc((size_t)(T > 0 ? T : 1), st));
        count_launch(), k_given_pairs<<<eg, 256, 0, st>>>(E, d_io.get(), d_ux.get(), d_vx.get(), d_ioff_old.get(),
                                          d_pairs_old.get(), d_flags.get());
    } else if (g->variant == DRESS_VARIANT_UNDIRECTED && !dup) {
        DevBuf<int> d_ocnt, d_otgt, d_oeid, d_osrc;
        DevBuf<long long> d_ooff;
        DevBuf<unsigned long long> d_cursor;
        DRESS_TRY(d_ocnt.alloc((size_t)N, st));
        DRESS_TRY(d_ooff.alloc((size_t)N + 1, st));
        DRESS_TRY(d_otgt.alloc((size_t)(S > 0 ? S : 1), st));
        DRESS_TRY(d_oeid.alloc((size_t)(S > 0 ? S : 1), st));
        DRESS_TRY(d_osrc.alloc((size_t)(S > 0 ? S : 1), st));
        const int vg = (int)grid_for(N, 256, 32 * sms);
        count_launch(), k_orient_count<<<vg, 256, 0, st>>>(N, d_off.get(), d_tgt.get(), d_deg.get(), d_ocnt.get());
        DRESS_TRY(exclusive_scan_i32(d_ocnt.get(), d_ooff.get(), N, d_scan_tmp.get(), st));
        count_launch(), k_orient_fill<<<vg, 256, 0, st>>>(N, d_off.get(), d_tgt.get(), d_eidx.get(), d_deg.get(),
                                          d_ooff.get(), d_otgt.get(), d_oeid.get(), d_osrc.get());
        long long M = 0;
        DRESS_CUDA_TRY(counted_memcpy(&M, d_ooff.get() + N, sizeof(M), cudaMemcpyDeviceToHost, st));
        DRESS_CUDA_TRY(cudaMemsetAsync(d_cnt.get(), 0, (size_t)E * sizeof(int), st));
        DRESS_CUDA_TRY(cudaStreamSynchronize(st));
        const int tg = (int)grid_for(M, 256, 64 * sms);
        count_launch(), k_triangles<false><<<tg, 256, 0, st>>>(M, d_ooff.get(), d_otgt.get(), d_oeid.get(), d_osrc.get(),
                                               d_cnt.get(), nullptr, nullptr);
        DRESS_TRY(exclusive_scan_i32(d_cnt.get(), d_ioff_old.get(), E, d_scan_tmp.get(), st));
        DRESS_CUDA_TRY(counted_memcpy(&T, d_ioff_old.get() + E, sizeof(T), cudaMemcpyDeviceToHost, st));
        DRESS_CUDA_TRY(cudaStreamSynchronize(st));
        DRESS_TRY(d_pairs_old.alloc((size_t)(T > 0 ? T : 1), st));
        DRESS_TRY(d_cursor.alloc((size_t)E, st));
        count_launch(), k_copy_i64<<<eg, 256, 0, st>>>(E, d_ioff_old.get(), d_cursor.get());
        count_launch(), k_triangles<true><<<tg, 256, 0, st>>>(M, d_ooff.get(), d_otgt.get(), d_oeid.get(), d_osrc.get(),
                                              nullptr, d_cursor.get(), d_pairs_old.get());
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
    d_tgt.release();

    // ---- bins and renumbering ---------------------------------------------------
    DevBuf<int> d_bc, d_vperm, d_vinv, d_eperm, d_einv;
    DRESS_TRY(d_bc.alloc(4 * NB, st));
    DRESS_TRY(d_vperm.alloc((size_t)N, st));
    DRESS_TRY(d_vinv.alloc((size_t)N, st));
    DRESS_TRY(d_eperm.alloc((size_t)E, st));
    DRESS_TRY(d_einv.alloc((size_t)E, st));
    DRESS_CUDA_TRY(cudaMemsetAsync(d_bc.get(), 0, 4 * NB * sizeof(int), st));
    const int vg = (int)grid_for(N, 256, 32 * sms);
    count_launch(), k_bin_count<<<vg, 256, 0, st>>>(N, d_deg.get(), 1, d_bc.get());
    count_launch(), k_bin_count<<<eg, 256, 0, st>>>(E, d_cnt.get(), 1, d_bc.get() + NB);
    int bc[2 * NB];
    DRESS_CUDA_TRY(counted_memcpy(bc, d_bc.get(), sizeof(bc), cudaMemcpyDeviceToHost, st));
    DRESS_CUDA_TRY(counted_memcpy(flags, d_flags.get(), sizeof(flags), cudaMemcpyDeviceToHost, st));
    DRESS_CUDA_TRY(cudaStreamSynchronize(st));
    if (flags[0]) return Status::Err(DRESSX_EINVAL, "malformed intercept tables");
    Bins vb, eb;
    vb.start[0] = eb.start[0] = 0;
    for (int b = 0; b < NB; ++b) {
        vb.start[b + 1] = vb.start[b] + bc[b];
        eb.start[b + 1] = eb.start[b] + bc[NB + b];
    }
    int cur[2 * NB];
    for (int b = 0; b < NB; ++b) { cur[b] = vb.start[b]; cur[NB + b] = eb.start[b]; }
    DRESS_CUDA_TRY(counted_memcpy(d_bc.get() + 2 * NB, cur, sizeof(cur), cudaMemcpyHostToDevice, st));
    count_launch(), k_bin_scatter<<<vg, 256, 0, st>>>(N, d_deg.get(), 1, d_bc.get() + 2 * NB, d_vperm.get(), d_vinv.get());
    count_launch(), k_bin_scatter<<<eg, 256, 0, st>>>(E, d_cnt.get(), 1, d_bc.get() + 3 * NB, d_eperm.get(), d_einv.get());

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
    DRESS_TRY(d_pairs.alloc((size_t)(T > 0 ? T : 1), st));
    count_launch(), k_new_pairs<<<eg, 256, 0, st>>>(E, d_eperm.get(), d_ioff_old.get(), d_pairs_old.get(), d_einv.get(),
                                    d_ioff.get(), d_pairs.get());
    DRESS_CUDA_TRY(cudaGetLastError());
    d_U.release(); d_V.release(); d_w.release(); d_d.release(); d_nw.release();
    d_pairs_old.release(); d_ioff_old.release(); d_ncnt.release(); d_cnt.release(); d_deg.release();

    // block-bin shared memory and spill area
    int smem_optin = 0;
    DRESS_CUDA_TRY(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, en.device));
    int block_cap = (smem_optin - 1024) / 8;
    // largest block-bin item (rows have max_row + 1 terms, edges at most that)
    long long big = 0;
    if (vb.start[BBLOCK + 1] > vb.start[BBLOCK] || eb.start[BBLOCK + 1] > eb.start[BBLOCK])
        big = max_row + 1;
    DevBuf<double> d_scratch;
    long long scratch_stride = 0;
    if (big > block_cap) {
        scratch_stride = big;
        DRESS_TRY(d_scratch.alloc((size_t)(2 * sms) * (size_t)big, st));
    }
    DRESS_CUDA_TRY(cudaFuncSetAttribute(k_vertex_block<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, block_cap * 8));
    DRESS_CUDA_TRY(cudaFuncSetAttribute(k_vertex_block<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, block_cap * 8));
    DRESS_CUDA_TRY(cudaFuncSetAttribute(k_edge_block<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, block_cap * 8));
    DRESS_CUDA_TRY(cudaFuncSetAttribute(k_edge_block<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, block_cap * 8));
    DRESS_CUDA_TRY(cudaFuncSetAttribute(k_vertex_warp<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 8 * WARP_CAP * 8));
    DRESS_CUDA_TRY(cudaFuncSetAttribute(k_vertex_warp<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 8 * WARP_CAP * 8));
    DRESS_CUDA_TRY(cudaFuncSetAttribute(k_edge_warp<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 8 * WARP_CAP * 8));
    DRESS_CUDA_TRY(cudaFuncSetAttribute(k_edge_warp<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 8 * WARP_CAP * 8));

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
    s.nw = d_nwi.get();
    s.ioff = d_ioff.get(); s.pairs = d_pairs.get();
    s.vd = d_vd.get(); s.maxd = d_maxd.get();
    s.eps = epsilon;
    s.scratch = d_scratch.get(); s.scratch_stride = scratch_stride;
    double *dbuf[2] = {d_dbuf.get(), d_dbuf.get() + E};
    double *pbuf[2] = {uniform ? nullptr : d_pbuf.get(), uniform ? nullptr : d_pbuf.get() + E};

    // per-sweep max|delta| slots form a ring; a chunk zeroes its own slots
    // first, and the first sweep of a chunk still sees the previous slot
    unsigned long long hmax[RING];
    int conv = -1, done = 0;
    int chunk = en.cfg.fit_chunk > 0 ? (en.cfg.fit_chunk < MAX_CHUNK ? en.cfg.fit_chunk : MAX_CHUNK) : 8;
    double last_delta = 0.0;
    while (done < max_iterations && conv < 0) {
        int hi = done + chunk < max_iterations ? done + chunk : max_iterations;
        for (int it = done; it < hi; ++it)
            DRESS_CUDA_TRY(cudaMemsetAsync(d_maxd.get() + it % RING, 0, sizeof(unsigned long long), st));
        for (int it = done; it < hi; ++it) {
            s.iter = it;
            s.slot = it % RING;
            s.prev_slot = (it + RING - 1) % RING;
            s.d = dbuf[it & 1]; s.dn = dbuf[(it + 1) & 1];
            s.p = pbuf[it & 1]; s.pn = pbuf[(it + 1) & 1];
            if (uniform) DRESS_TRY(launch_sweep<true>(s, vb, eb, sms, block_cap, st));
            else         DRESS_TRY(launch_sweep<false>(s, vb, eb, sms, block_cap, st));
        }
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
        if (chunk < 32) chunk *= 2;
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
    count_launch(), k_unpermute<<<eg, 256, 0, st>>>(E, d_eperm.get(), dbuf[(last + 1) & 1], d_out.get());
    count_launch(), k_unpermute<<<vg, 256, 0, st>>>(N, d_vperm.get(), d_vd.get(), d_out.get() + E);
    if (E > 0)
        DRESS_CUDA_TRY(counted_memcpy(g->edge_dress, d_out.get(), (size_t)E * sizeof(double),
                                       cudaMemcpyDeviceToHost, st));
    if (N > 0)
        DRESS_CUDA_TRY(counted_memcpy(g->vertex_dress, d_out.get() + E, (size_t)N * sizeof(double),
                                       cudaMemcpyDeviceToHost, st));
    DRESS_CUDA_TRY(cudaStreamSynchronize(st));
    if (iterations) *iterations = conv >= 0 ? conv : max_iterations;
    if (delta) *delta = last_delta;
    if (stats) {
        stats->T = T;
        stats->sweeps = last + 1;
        stats->setup_ms = setup_ms;
        stats->iterate_ms = sweep_ms;
    }
    return Status::Ok();
}

}  // namespace dress
