// sweep.cuh -- the per-sweep kernels of the single-graph fit (fit_graph.cu).
//
// Reference: libdress/src/dress.c:556-591 (vertex norms, edge update) with
// the sorted KBN sum of dress.c:51-66.
//
// Items (vertices, edges) are binned by their number of STORED terms: the
// row's slots for a vertex, the common-neighbour pairs for an edge.  Every
// item has one more term, its self term (4*nw for a vertex, the self/own-edge
// term for an edge), which is merged into the sorted sequence at its rank.
//
// Persistent order: the storage order of a row's slots (row_eid) and of an
// edge's pairs is irrelevant to the result (the sum sorts its terms), so each
// sweep keeps them in the order of the previous sweep's values.  A sweep
// gathers the terms in stored order, checks that they are ascending, and only
// when they are not sorts them (carrying the slot / pair along) and writes the
// new order back.  Once the values settle, most items skip the sort.
//
//   bins: 0 stored terms; <=2, <=4, <=8, <=16 (one thread per item, register
//   network); <=MED_CAP (one thread per item streaming its terms: the sum runs
//   while the order is checked; an item found out of order is queued, sorted
//   by a warp and streamed again); more (one block per item, shared memory,
//   largest items first; rows beyond the shared capacity spill to a global
//   slab).  The block items are split at BIG_CAP so that the smaller ones run
//   several blocks per SM.
#pragma once
#include <algorithm>
#include <climits>

#include "common.cuh"
#include "engine.h"

namespace dress {
namespace sweep {

constexpr int NB = 8;
constexpr int MED_CAP = 512;        // stored terms of a streamed (one-thread) item
constexpr int BIG_CAP = 4096;       // block items up to this share an SM
enum { B0 = 0, B2, B4, B8, B16, BMED, BBLOCK, BBIG };

__host__ __device__ __forceinline__ int bin_of(long long n)
{
    return n == 0 ? B0 : n <= 2 ? B2 : n <= 4 ? B4 : n <= 8 ? B8 : n <= 16 ? B16 : n <= MED_CAP ? BMED
         : n <= BIG_CAP ? BBLOCK : BBIG;
}

// Fine keys of the renumbering: the coarse bins, with the streamed bin split
// by exact term count, longest first -- neighbouring threads then run loops
// of equal length, and the longest loops start first.
constexpr int NF = BMED + (MED_CAP - 16) + 2;

__host__ __device__ __forceinline__ int fine_of(long long n)
{
    const int b = bin_of(n);
    if (b < BMED) return b;
    if (b == BMED) return BMED + (MED_CAP - (int)n);
    return BMED + (MED_CAP - 16) + (b - BBLOCK);
}

// first fine key of a coarse bin
__host__ __device__ __forceinline__ int fine_first(int b)
{
    return b <= BMED ? b : BMED + (MED_CAP - 16) + (b - BBLOCK);
}

struct Sweep {
    int N, E, fwd;                 // fwd: FORWARD/BACKWARD self term
    const long long *row_off;      // [N+1] renumbered CSR rows
    int *row_eid;                  // [S]  slot edge ids, kept in value order
    const int *eu, *ev;            // [E]
    const double *w;               // [E] (weighted graphs)
    double wc;                     // the weight when all are equal
    const double *nw;              // [N], or null when every vertex weight is 1.0
    const long long *ioff;         // [E+1]
    int2 *pairs;                   // [T]  common-neighbour edge pairs, kept in value order
    double *vd;                    // [N]
    unsigned long long *maxd;      // convergence ring
    const double *d, *p;           // current values and products
    double *dn, *pn;               // next values and products
    const int *iter;               // device: index of the sweep being run
    int max_iter;                  // sweeps at or past it return at once
    double eps;
    double *scratch_k;             // block-bin spill (keys), per block
    int2 *scratch_v;               // block-bin spill (payload), per block
    long long scratch_stride;
    int *qv, *qe;                  // streamed items found out of order (vertices, edges)
    unsigned *qcount;              // [2] queue lengths
    double *bkey_v, *bkey_e;       // sorted terms of the block items, one slot per item
    const long long *bofs_v, *bofs_e;   // slot offsets, indexed from bv0 / be0
    int bv0, be0;                  // first block item (vertex, edge)
    double *skey, *tkey;           // sorted terms of queued streamed items, at their
    long long sbase, tbase;        // row slot / pair offset minus these bases
};

// Per-sweep max|delta| slots form a ring; the sweep index lives in device
// memory, so every sweep of a chunk is the same launch sequence (replayed from
// a CUDA graph) and the sweeps after convergence return at once.
constexpr int RING = 64;

__device__ __forceinline__ bool skipped(const Sweep &s)
{
    const int it = *s.iter;
    return it >= s.max_iter ||
           (it > 0 && __longlong_as_double((long long)s.maxd[(it + RING - 1) % RING]) < s.eps);
}

__device__ __forceinline__ unsigned long long *max_slot(const Sweep &s) { return &s.maxd[*s.iter % RING]; }

// end of a sweep: the next index, its slot cleared
__global__ void k_next_sweep(int *iter, unsigned long long *maxd)
{
    const int it = *iter + 1;
    *iter = it;
    maxd[it % RING] = 0ULL;
}

template <bool UNIF>
__device__ __forceinline__ double prod(const Sweep &s, int e)
{
    return UNIF ? dmul(s.wc, s.d[e]) : s.p[e];
}

// 4 * nw of a vertex (exactly 4.0 for unit weights)
__device__ __forceinline__ double four_nw(const Sweep &s, int i)
{
    return s.nw ? dmul(4.0, s.nw[i]) : 4.0;
}

template <bool UNIF>
__device__ __forceinline__ double self_term(const Sweep &s, int j, int u, int v)
{
    double own = prod<UNIF>(s, j);
    double a = four_nw(s, u);
    if (s.fwd) return dadd(a, own);
    return dadd(dadd(a, four_nw(s, v)), dmul(2.0, own));
}

// edge value from its numerator; stores d_next (and p_next), returns |delta|
template <bool UNIF>
__device__ __forceinline__ double finish_edge(const Sweep &s, int j, int u, int v, double num)
{
    double den = dmul(s.vd[u], s.vd[v]);
    double r = den > 0.0 ? ddiv(num, den) : 0.0;
    s.dn[j] = r;
    if (!UNIF) s.pn[j] = dmul(s.w[j], r);
    return fabs(dsub(s.d[j], r));
}

// ---- register helpers -------------------------------------------------------------

template <class P>
__device__ __forceinline__ void cswap_kv(double &a, double &b, P &x, P &y)
{
    bool sw = b < a;
    double lo = sw ? b : a, hi = sw ? a : b;
    P plo = sw ? y : x, phi = sw ? x : y;
    a = lo; b = hi; x = plo; y = phi;
}

// single-direction bitonic network on M registers, payload carried along
template <int M, class P>
__device__ __forceinline__ void sort_kv(double (&a)[M], P (&v)[M])
{
#pragma unroll
    for (int k = 2; k <= M; k <<= 1) {
#pragma unroll
        for (int i = 0; i < M; ++i) {
            int j = i ^ (k - 1);
            if (j > i) cswap_kv(a[i], a[j], v[i], v[j]);
        }
#pragma unroll
        for (int st = k >> 2; st > 0; st >>= 1) {
#pragma unroll
            for (int i = 0; i < M; ++i) {
                int j = i ^ st;
                if (j > i) cswap_kv(a[i], a[j], v[i], v[j]);
            }
        }
    }
}

// Sorted KBN of a[0..n) (ascending, n <= M) with x merged in at its rank.
template <int M>
__device__ __forceinline__ double kbn_merge_regs(const double (&a)[M], int n, double x)
{
    int pos = 0;
#pragma unroll
    for (int k = 0; k < M; ++k) pos += (k < n && a[k] < x);
    double s = pos == 0 ? x : a[0], c = 0.0;
#pragma unroll
    for (int t = 1; t <= M; ++t) {
        if (t <= n) {
            double v = t < pos ? a[t < M ? t : M - 1] : (t == pos ? x : a[t - 1]);
            kbn_step(s, c, v);
        }
    }
    return dadd(s, c);
}

// Sorted KBN of an ascending stream with one extra term x merged at its
// rank (x goes before the first term >= x, exactly where kbn_merge_buf puts it).
struct KbnStream {
    double s, c, x;
    bool started, inserted;
    __device__ __forceinline__ explicit KbnStream(double extra) : s(0.0), c(0.0), x(extra), started(false), inserted(false) {}
    __device__ __forceinline__ void raw(double v)
    {
        if (started) kbn_step(s, c, v);
        else { s = v; started = true; }
    }
    __device__ __forceinline__ void push(double v)
    {
        if (!inserted && !(v < x)) { raw(x); inserted = true; }
        raw(v);
    }
    __device__ __forceinline__ double finish()
    {
        if (!inserted) raw(x);
        return dadd(s, c);
    }
};

// KBN steps over a[b..e) in index order, in W-term windows: the next
// window's loads are in flight while the current one is summed, and the
// ragged tail is loaded at once, so the chain does not wait on L2 or HBM
// term by term.
__device__ __forceinline__ void kbn_run(const double *__restrict__ a, int b, int e, double &s, double &c)
{
    constexpr int W = 32;
    int i = b;
    if (i + W <= e) {
        double cur[W], nxt[W];
#pragma unroll
        for (int t = 0; t < W; ++t) cur[t] = a[i + t];
        while (i + 2 * W <= e) {
#pragma unroll
            for (int t = 0; t < W; ++t) nxt[t] = a[i + W + t];
#pragma unroll
            for (int t = 0; t < W; ++t) kbn_step(s, c, cur[t]);
#pragma unroll
            for (int t = 0; t < W; ++t) cur[t] = nxt[t];
            i += W;
        }
#pragma unroll
        for (int t = 0; t < W; ++t) kbn_step(s, c, cur[t]);
        i += W;
    }
    if (i < e) {
        double tail[W];
#pragma unroll
        for (int t = 0; t < W; ++t) tail[t] = i + t < e ? a[i + t] : 0.0;
#pragma unroll
        for (int t = 0; t < W; ++t)
            if (i + t < e) kbn_step(s, c, tail[t]);
    }
}

// Same over an ascending run in global memory: the self term's rank by
// binary search, then the windowed steps before it, the self term, and the
// windowed steps after it.
__device__ __forceinline__ double kbn_merge_stream(const double *__restrict__ a, int n, double x)
{
    int lo = 0, hi = n;                      // first index with a[idx] >= x
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (a[mid] < x) lo = mid + 1;
        else hi = mid;
    }
    const int pos = lo;
    // s = -0.0, c = +0.0: the first step then leaves s = that term, c = +0.0
    // exactly, as starting the sum at it does (for every finite term, zeros
    // of either sign included)
    double s = -0.0, c = 0.0;
    kbn_run(a, 0, pos, s, c);
    kbn_step(s, c, x);
    kbn_run(a, pos, n, s, c);
    return dadd(s, c);
}

// ---- asynchronous global -> shared copies (cp.async, 8 bytes a thread) ----------------
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_one() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// Same as kbn_merge_stream for one long run, by a whole warp: the lanes copy
// chunks of HUB_CHUNK terms into shared memory (buf, 2 x HUB_CHUNK doubles)
// one chunk ahead of lane 0, which runs the serial chain from shared memory.
// The result is valid in lane 0.
constexpr int HUB_CHUNK = 1024;
constexpr size_t HUB_SMEM = 2 * HUB_CHUNK * sizeof(double);
__device__ __forceinline__ double kbn_merge_stream_warp(const double *__restrict__ a, int n, double x, double *buf,
                                                        int lane)
{
    int pos = 0;
    if (lane == 0) {
        int lo = 0, hi = n;                  // first index with a[idx] >= x
        while (lo < hi) {
            int mid = (lo + hi) >> 1;
            if (a[mid] < x) lo = mid + 1;
            else hi = mid;
        }
        pos = lo;
    }
    pos = __shfl_sync(0xffffffffu, pos, 0);
    const int nch = (n + HUB_CHUNK - 1) / HUB_CHUNK;
    auto issue = [&](int ch) {
        if (ch < nch) {
            const int base = ch * HUB_CHUNK;
            double *dst = buf + (ch & 1) * HUB_CHUNK;
            for (int t = lane; t < HUB_CHUNK && base + t < n; t += 32) cp_async8(dst + t, a + base + t);
        }
        cp_async_commit();                   // one group per chunk on every lane, empty or not
    };
    double s = -0.0, c = 0.0;                // see kbn_merge_stream
    issue(0);
    for (int ch = 0; ch < nch; ++ch) {
        issue(ch + 1);
        cp_async_wait_one();                 // this lane's copies of chunk ch landed ...
        __syncwarp();                        // ... and every lane's
        if (lane == 0) {
            const double *src = buf + (ch & 1) * HUB_CHUNK;
            const int base = ch * HUB_CHUNK, cnt = min(HUB_CHUNK, n - base);
            const int cut = min(max(pos - base, 0), cnt);     // terms of this chunk before x
            int t = 0;
            for (; t + 8 <= cut; t += 8) {
                double v[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) v[q] = src[t + q];
#pragma unroll
                for (int q = 0; q < 8; ++q) kbn_step(s, c, v[q]);
            }
            for (; t < cut; ++t) kbn_step(s, c, src[t]);
            if (pos >= base && pos < base + cnt) kbn_step(s, c, x);
            for (; t + 8 <= cnt; t += 8) {
                double v[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) v[q] = src[t + q];
#pragma unroll
                for (int q = 0; q < 8; ++q) kbn_step(s, c, v[q]);
            }
            for (; t < cnt; ++t) kbn_step(s, c, src[t]);
        }
        __syncwarp();                        // chunk ch read before its buffer is refilled
    }
    if (pos == n) kbn_step(s, c, x);
    return dadd(s, c);
}

// Sorted KBN of the n terms term(0..n) taken in stored order, with x merged
// at its rank, while checking that the terms ascend; false, without
// finishing, at the first window that does not ascend.  Windows of W terms,
// the next window gathered while the current one is summed; x is looked for
// once per window; the ragged tail is gathered at once.
template <int W, class Term>
__device__ __forceinline__ bool kbn_stream_checked(int n, double x, Term term, double &out)
{
    double s = -0.0, c = 0.0, prev = -DRESS_INF;     // see kbn_merge_stream
    bool ins = false, ok = true;
    int i = 0;
    if (n >= W) {
        double cur[W], nxt[W];
#pragma unroll
        for (int t = 0; t < W; ++t) cur[t] = term(t);
        for (;;) {
            const bool more = i + 2 * W <= n;
            if (more) {
#pragma unroll
                for (int t = 0; t < W; ++t) nxt[t] = term(i + W + t);
            }
            bool o = !(cur[0] < prev);
#pragma unroll
            for (int t = 0; t + 1 < W; ++t) o &= !(cur[t + 1] < cur[t]);
            if (!o) return false;        // out of order: the item is sorted and summed elsewhere
            prev = cur[W - 1];
            if (!ins && !(cur[W - 1] < x)) {
#pragma unroll
                for (int t = 0; t < W; ++t) {
                    if (!ins && !(cur[t] < x)) {
                        kbn_step(s, c, x);
                        ins = true;
                    }
                    kbn_step(s, c, cur[t]);
                }
            } else {
#pragma unroll
                for (int t = 0; t < W; ++t) kbn_step(s, c, cur[t]);
            }
            i += W;
            if (!more) break;
#pragma unroll
            for (int t = 0; t < W; ++t) cur[t] = nxt[t];
        }
    }
    if (i < n) {
        // the ragged tail, its terms loaded at once
        double tail[W];
#pragma unroll
        for (int t = 0; t < W; ++t) tail[t] = i + t < n ? term(i + t) : 0.0;
#pragma unroll
        for (int t = 0; t < W; ++t)
            if (i + t < n) {
                ok &= !(tail[t] < prev);
                prev = tail[t];
            }
        if (!ok) return false;
#pragma unroll
        for (int t = 0; t < W; ++t)
            if (i + t < n) {
                if (!ins && !(tail[t] < x)) {
                    kbn_step(s, c, x);
                    ins = true;
                }
                kbn_step(s, c, tail[t]);
            }
    }
    if (!ins) kbn_step(s, c, x);
    out = dadd(s, c);
    return true;
}

// Same over an ascending buffer (one thread).
__device__ __forceinline__ double kbn_merge_buf(const double *a, int n, double x)
{
    int lo = 0, hi = n;                      // first index with a[idx] >= x
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (a[mid] < x) lo = mid + 1;
        else hi = mid;
    }
    const int pos = lo;
    double s, c = 0.0;
    int i;
    if (pos == 0) {
        s = x;
        i = 0;
    } else {
        s = a[0];
        for (i = 1; i < pos; ++i) kbn_step(s, c, a[i]);
        kbn_step(s, c, x);
    }
    // 8-term windows, the next window loaded while the current one is summed
    if (i + 8 <= n) {
        double cur[8], nxt[8];
#pragma unroll
        for (int t = 0; t < 8; ++t) cur[t] = a[i + t];
        while (i + 16 <= n) {
#pragma unroll
            for (int t = 0; t < 8; ++t) nxt[t] = a[i + 8 + t];
#pragma unroll
            for (int t = 0; t < 8; ++t) kbn_step(s, c, cur[t]);
#pragma unroll
            for (int t = 0; t < 8; ++t) cur[t] = nxt[t];
            i += 8;
        }
#pragma unroll
        for (int t = 0; t < 8; ++t) kbn_step(s, c, cur[t]);
        i += 8;
    }
    for (; i < n; ++i) kbn_step(s, c, a[i]);
    return dadd(s, c);
}

// Cooperative ascending sort of keys[0..n) with payload (warp or block).
template <class P, class Sync>
__device__ __forceinline__ void sort_shared_kv(double *keys, P *vals, int n, int tid, int nthr, Sync sync)
{
    int M = 1;
    while (M < n) M <<= 1;
    for (int k = 2; k <= M; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            const int half = M >> 1;
            for (int q = tid; q < half; q += nthr) {
                int i = ((q & ~(j - 1)) << 1) | (q & (j - 1));
                int p = (j == (k >> 1)) ? (i ^ (k - 1)) : (i | j);
                int lo = i < p ? i : p, hi = i < p ? p : i;
                if (hi < n) {
                    double x = keys[lo], y = keys[hi];
                    if (y < x) {
                        keys[lo] = y;
                        keys[hi] = x;
                        P t = vals[lo];
                        vals[lo] = vals[hi];
                        vals[hi] = t;
                    }
                }
            }
            sync();
        }
    }
}

struct WarpSync { __device__ void operator()() const { __syncwarp(); } };
struct BlockSync { __device__ void operator()() const { __syncthreads(); } };
struct WarpAny { __device__ bool operator()(bool p) const { return __any_sync(0xffffffffu, p); } };
struct BlockAny { __device__ bool operator()(bool p) const { return __syncthreads_or(p) != 0; } };

// Restores ascending order of a nearly sorted keys[0..n) (payload carried):
// odd-even transposition passes until one pass swaps nothing -- as many passes
// as the farthest displacement -- and a full bitonic sort if that takes more
// than MAX_PASSES passes.  Ends with all cooperating threads synchronised.
constexpr int MAX_PASSES = 16;

// fraction of descents above which the odd-even passes are skipped
__device__ __forceinline__ bool far_from_sorted(int descents, int n) { return 8 * descents > n; }
template <class P, class Sync, class Any>
__device__ __forceinline__ void fix_order(double *keys, P *vals, int n, int tid, int nthr, Sync sync, Any any,
                                          bool far = false)
{
    for (int pass = 0; pass < MAX_PASSES && !far; ++pass) {
        bool sw = false;
        for (int parity = 0; parity < 2; ++parity) {
            for (int i = 2 * tid + parity; i + 1 < n; i += 2 * nthr) {
                double x = keys[i], y = keys[i + 1];
                if (y < x) {
                    keys[i] = y;
                    keys[i + 1] = x;
                    P t = vals[i];
                    vals[i] = vals[i + 1];
                    vals[i + 1] = t;
                    sw = true;
                }
            }
            sync();
        }
        if (!any(sw)) return;
    }
    sort_shared_kv(keys, vals, n, tid, nthr, sync);
}

// ---- one thread per item (at most 16 stored terms) ----------------------------------

// Grid-stride loops over a bounded grid: one convergence atomic per block,
// not one per 128 items.
template <int M, bool UNIF>
__global__ void __launch_bounds__(128) k_vertex_thr(Sweep s, int begin, int end)
{
    if (skipped(s)) return;
    for (int i = begin + blockIdx.x * blockDim.x + threadIdx.x; i < end; i += gridDim.x * blockDim.x) {
        const double self = four_nw(s, i);
        if constexpr (M == 0) {
            s.vd[i] = dsqrt(dadd(self, 0.0));
        } else {
            const long long b = s.row_off[i];
            const int deg = (int)(s.row_off[i + 1] - b);
            double a[M];
            int id[M];
#pragma unroll
            for (int k = 0; k < M; ++k) {
                if (k < deg) {
                    id[k] = s.row_eid[b + k];
                    a[k] = prod<UNIF>(s, id[k]);
                } else {
                    id[k] = -1;
                    a[k] = DRESS_INF;
                }
            }
            bool sorted = true;
#pragma unroll
            for (int k = 0; k + 1 < M; ++k) sorted &= !(a[k + 1] < a[k]);
            if (!sorted) {
                sort_kv<M>(a, id);
#pragma unroll
                for (int k = 0; k < M; ++k)
                    if (k < deg) s.row_eid[b + k] = id[k];
            }
            s.vd[i] = dsqrt(kbn_merge_regs<M>(a, deg, self));
        }
    }
}

template <int M, bool UNIF>
__global__ void __launch_bounds__(128) k_edge_thr(Sweep s, int begin, int end)
{
    if (skipped(s)) return;
    double delta = 0.0;
    for (int j = begin + blockIdx.x * blockDim.x + threadIdx.x; j < end; j += gridDim.x * blockDim.x) {
        const int u = s.eu[j], v = s.ev[j];
        const double self = self_term<UNIF>(s, j, u, v);
        double num;
        if constexpr (M == 0) {
            num = dadd(self, 0.0);               // sorted KBN of the single self term
        } else {
            const long long o = s.ioff[j];
            const int nc = (int)(s.ioff[j + 1] - o);
            double a[M];
            int2 id[M];
#pragma unroll
            for (int k = 0; k < M; ++k) {
                if (k < nc) {
                    id[k] = s.pairs[o + k];
                    a[k] = dadd(prod<UNIF>(s, id[k].x), prod<UNIF>(s, id[k].y));
                } else {
                    id[k] = make_int2(-1, -1);
                    a[k] = DRESS_INF;
                }
            }
            bool sorted = true;
#pragma unroll
            for (int k = 0; k + 1 < M; ++k) sorted &= !(a[k + 1] < a[k]);
            if (!sorted) {
                sort_kv<M>(a, id);
#pragma unroll
                for (int k = 0; k < M; ++k)
                    if (k < nc) s.pairs[o + k] = id[k];
            }
            num = kbn_merge_regs<M>(a, nc, self);
        }
        delta = fmax(delta, finish_edge<UNIF>(s, j, u, v, num));
    }
    block_max_to(max_slot(s), delta);
}

// ---- one thread per item, streamed (at most MED_CAP stored terms) ---------------------
// The terms are gathered STREAM_D at a time (independent loads in flight),
// summed in stored order while the order is checked; an item met out of
// order is queued for k_*_med_sort, which sorts it and finishes it.
constexpr int STREAM_D = 16;

template <bool UNIF>
__global__ void __launch_bounds__(256) k_vertex_med(Sweep s, int begin, int end)
{
    if (skipped(s)) return;
    for (int i = begin + blockIdx.x * blockDim.x + threadIdx.x; i < end; i += gridDim.x * blockDim.x) {
        const long long b = s.row_off[i];
        const int deg = (int)(s.row_off[i + 1] - b);
        const int *rows = s.row_eid + b;
        double sum;
        if (kbn_stream_checked<STREAM_D>(deg, four_nw(s, i), [&](int k) { return prod<UNIF>(s, rows[k]); }, sum))
            s.vd[i] = dsqrt(sum);
        else
            s.qv[atomicAdd(&s.qcount[0], 1u)] = i;
    }
}

template <bool UNIF>
__global__ void __launch_bounds__(256) k_edge_med(Sweep s, int begin, int end)
{
    if (skipped(s)) return;
    double delta = 0.0;
    for (int j = begin + blockIdx.x * blockDim.x + threadIdx.x; j < end; j += gridDim.x * blockDim.x) {
        const int u = s.eu[j], v = s.ev[j];
        const long long o = s.ioff[j];
        const int nc = (int)(s.ioff[j + 1] - o);
        const int2 *prs = s.pairs + o;
        double sum;
        if (kbn_stream_checked<STREAM_D>(nc, self_term<UNIF>(s, j, u, v), [&](int k) {
                const int2 pr = prs[k];
                return dadd(prod<UNIF>(s, pr.x), prod<UNIF>(s, pr.y));
            }, sum))
            delta = fmax(delta, finish_edge<UNIF>(s, j, u, v, sum));
        else
            s.qe[atomicAdd(&s.qcount[1], 1u)] = j;
    }
    block_max_to(max_slot(s), delta);
}

// ---- packed warp sort of one queued streamed item --------------------------------------
// The terms are sorted as 64-bit words: the term's order-preserving bits with
// the low IDX_BITS replaced by its stored position, the replaced bits kept
// beside it (lo, by position).  Words are distinct, so the sort is total, and
// moving a word moves key and position together: no payload array in shared
// memory, half the traffic of sorting keys with a payload, and more warps
// per SM.  Afterwards the payload (slot edge id or pair) is gathered by
// position.  Terms equal in all but their low IDX_BITS come out in stored
// order, so the order of the full values is checked and, where such a near
// tie is inverted (rare), repaired.
constexpr int IDX_BITS = 9;
constexpr unsigned long long IDX_MASK = (1ULL << IDX_BITS) - 1;
static_assert(MED_CAP <= (1 << IDX_BITS), "positions must fit the index bits");

// order-preserving map of a double to 64 unsigned bits, and back
__device__ __forceinline__ unsigned long long ord_bits(double x)
{
    const unsigned long long u = (unsigned long long)__double_as_longlong(x);
    return u ^ ((u >> 63) ? ~0ULL : 0x8000000000000000ULL);
}
__device__ __forceinline__ double from_ord(unsigned long long k)
{
    return __longlong_as_double((long long)(k ^ ((k >> 63) ? 0x8000000000000000ULL : ~0ULL)));
}

__device__ __forceinline__ void pack_term(unsigned long long *wb, unsigned short *lo, int k, double v)
{
    const unsigned long long b = ord_bits(v);
    wb[k] = (b & ~IDX_MASK) | (unsigned long long)k;
    lo[k] = (unsigned short)(b & IDX_MASK);
}

// warp bitonic sort of w[0..n), the network of sort_shared
__device__ __forceinline__ void sort_words(unsigned long long *w, int n, int lane)
{
    int M = 1;
    while (M < n) M <<= 1;
    for (int k = 2; k <= M; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int q = lane; q < (M >> 1); q += 32) {
                const int i = ((q & ~(j - 1)) << 1) | (q & (j - 1));
                const int p = (j == (k >> 1)) ? (i ^ (k - 1)) : (i | j);
                const int a = i < p ? i : p, b = i < p ? p : i;
                if (b < n) {
                    const unsigned long long x = w[a], y = w[b];
                    if (y < x) {
                        w[a] = y;
                        w[b] = x;
                    }
                }
            }
            __syncwarp();
        }
    }
}

// Ascending order of w[0..n): odd-even transposition passes while they last
// at most MAX_PASSES (nearly sorted input), else the bitonic sort.
__device__ __forceinline__ void fix_words(unsigned long long *w, int n, int lane)
{
    int d = 0;
    for (int k = lane; k + 1 < n; k += 32) d += w[k + 1] < w[k];
    for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
    if (!far_from_sorted(d, n)) {
        for (int pass = 0; pass < MAX_PASSES; ++pass) {
            bool sw = false;
            for (int parity = 0; parity < 2; ++parity) {
                for (int i = 2 * lane + parity; i + 1 < n; i += 64) {
                    const unsigned long long x = w[i], y = w[i + 1];
                    if (y < x) {
                        w[i] = y;
                        w[i + 1] = x;
                        sw = true;
                    }
                }
                __syncwarp();
            }
            if (!__any_sync(0xffffffffu, sw)) return;
        }
    }
    sort_words(w, n, lane);
}

// Sorted words back to terms: the sorted values to out[0..n), the payload
// pay[0..n) (global, in stored order) permuted to the sorted order in place,
// parked in out on the way (every read of pay precedes every write).
template <class P>
__device__ __forceinline__ long long payload_bits(P v)
{
    long long b = 0;
    memcpy(&b, &v, sizeof(P));
    return b;
}
template <class P>
__device__ __forceinline__ P payload_of(long long b)
{
    P v;
    memcpy(&v, &b, sizeof(P));
    return v;
}

template <class P>
__device__ __forceinline__ void place_sorted(unsigned long long *wb, const unsigned short *lo, int n, int lane,
                                             P *pay, double *out)
{
    static_assert(sizeof(P) <= sizeof(double), "payload parks in a value slot");
    for (int k = lane; k < n; k += 32)
        out[k] = __longlong_as_double(payload_bits(pay[(int)(wb[k] & IDX_MASK)]));
    __syncwarp();
    for (int k = lane; k < n; k += 32) {
        const unsigned long long w = wb[k];
        const unsigned long long full = (w & ~IDX_MASK) | lo[(int)(w & IDX_MASK)];
        pay[k] = payload_of<P>(__double_as_longlong(out[k]));
        out[k] = from_ord(full);
        wb[k] = full;
    }
    __syncwarp();
    bool desc = false;
    for (int k = lane; k + 1 < n; k += 32) desc |= wb[k + 1] < wb[k];
    if (__any_sync(0xffffffffu, desc)) {
        // an inverted near tie: insertion by the full value, one lane
        if (lane == 0) {
            for (int k = 1; k < n; ++k) {
                const unsigned long long key = wb[k];
                const P pk = pay[k];
                int m = k - 1;
                while (m >= 0 && key < wb[m]) {
                    wb[m + 1] = wb[m];
                    pay[m + 1] = pay[m];
                    --m;
                }
                wb[m + 1] = key;
                pay[m + 1] = pk;
            }
            for (int k = 0; k < n; ++k) out[k] = from_ord(wb[k]);
        }
        __syncwarp();
    }
}

// one warp per queued item: restore ascending order, write it back with the
// sorted terms; the sums follow (k_*_med_sum) -- queued items are the minority
template <bool UNIF>
__global__ void __launch_bounds__(256) k_vertex_med_sort(Sweep s)
{
    extern __shared__ __align__(16) unsigned char smw[];
    if (skipped(s)) return;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    unsigned long long *wb = (unsigned long long *)smw + (size_t)wid * MED_CAP;
    unsigned short *lo = (unsigned short *)((unsigned long long *)smw + (size_t)nwarps * MED_CAP) +
                         (size_t)wid * MED_CAP;
    const int n_items = (int)s.qcount[0];
    for (int q = blockIdx.x * nwarps + wid; q < n_items; q += gridDim.x * nwarps) {
        const int i = s.qv[q];
        const long long b = s.row_off[i];
        const int deg = (int)(s.row_off[i + 1] - b);
        int *rows = s.row_eid + b;
#pragma unroll 4
        for (int k = lane; k < deg; k += 32) pack_term(wb, lo, k, prod<UNIF>(s, rows[k]));
        __syncwarp();
        fix_words(wb, deg, lane);
        place_sorted(wb, lo, deg, lane, rows, s.skey + (b - s.sbase));
    }
}

template <bool UNIF>
__global__ void __launch_bounds__(256) k_edge_med_sort(Sweep s)
{
    extern __shared__ __align__(16) unsigned char smw[];
    if (skipped(s)) return;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    unsigned long long *wb = (unsigned long long *)smw + (size_t)wid * MED_CAP;
    unsigned short *lo = (unsigned short *)((unsigned long long *)smw + (size_t)nwarps * MED_CAP) +
                         (size_t)wid * MED_CAP;
    const int n_items = (int)s.qcount[1];
    for (int q = blockIdx.x * nwarps + wid; q < n_items; q += gridDim.x * nwarps) {
        const int j = s.qe[q];
        const long long o = s.ioff[j];
        const int nc = (int)(s.ioff[j + 1] - o);
        int2 *prs = s.pairs + o;
#pragma unroll 4
        for (int k = lane; k < nc; k += 32) {
            const int2 pr = prs[k];
            pack_term(wb, lo, k, dadd(prod<UNIF>(s, pr.x), prod<UNIF>(s, pr.y)));
        }
        __syncwarp();
        fix_words(wb, nc, lane);
        place_sorted(wb, lo, nc, lane, prs, s.tkey + (o - s.tbase));
    }
}

// one thread per queued item: the sequential sum of its sorted terms
template <bool UNIF>
__global__ void __launch_bounds__(128) k_vertex_med_sum(Sweep s)
{
    if (skipped(s)) return;
    const int n_items = (int)s.qcount[0];
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n_items; q += gridDim.x * blockDim.x) {
        const int i = s.qv[q];
        const long long b = s.row_off[i];
        const int deg = (int)(s.row_off[i + 1] - b);
        s.vd[i] = dsqrt(kbn_merge_stream(s.skey + (b - s.sbase), deg, four_nw(s, i)));
    }
}

template <bool UNIF>
__global__ void __launch_bounds__(128) k_edge_med_sum(Sweep s)
{
    if (skipped(s)) return;
    double delta = 0.0;
    const int n_items = (int)s.qcount[1];
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n_items; q += gridDim.x * blockDim.x) {
        const int j = s.qe[q];
        const long long o = s.ioff[j];
        const int nc = (int)(s.ioff[j + 1] - o);
        const int u = s.eu[j], v = s.ev[j];
        delta = fmax(delta, finish_edge<UNIF>(s, j, u, v, kbn_merge_stream(s.tkey + (o - s.tbase), nc,
                                                                          self_term<UNIF>(s, j, u, v))));
    }
    block_max_to(max_slot(s), delta);
}

// ---- one block per item (hub rows, hub edges) -----------------------------------------
// The block gathers the item's terms in stored order, restores ascending
// order when needed (writing the new order back), and stores the sorted terms
// in the item's slot of bkey_*; the sequential sums run afterwards, one thread
// per item (k_*_block_sum), so no block idles behind a single summing thread.
// Items beyond the shared capacity are sorted in place in their slot.

template <bool UNIF, bool SUM_HERE>
__global__ void __launch_bounds__(512) k_vertex_block(Sweep s, int begin, int end, int cap)   // cap: 12 B per term
{
    extern __shared__ __align__(16) unsigned char smb[];
    __shared__ int descents;
    if (skipped(s)) return;
    for (int i = begin + blockIdx.x; i < end; i += gridDim.x) {
        const long long b = s.row_off[i];
        const int deg = (int)(s.row_off[i + 1] - b);
        double *slot = s.bkey_v + s.bofs_v[i - s.bv0];
        const bool inshm = deg <= cap;
        double *kb = inshm ? (double *)smb : slot;
        int *pb = inshm ? (int *)((double *)smb + cap) : (int *)(s.scratch_v + (long long)blockIdx.x * s.scratch_stride);
        if (threadIdx.x == 0) descents = 0;
        for (int k = threadIdx.x; k < deg; k += blockDim.x) {
            int e = s.row_eid[b + k];
            pb[k] = e;
            kb[k] = prod<UNIF>(s, e);
        }
        __syncthreads();
        int d = 0;
        for (int k = threadIdx.x; k + 1 < deg; k += blockDim.x) d += kb[k + 1] < kb[k];
        if (d) atomicAdd(&descents, d);
        __syncthreads();
        const int nd = descents;
        if (nd) {
            fix_order(kb, pb, deg, threadIdx.x, blockDim.x, BlockSync(), BlockAny(), far_from_sorted(nd, deg));
            for (int k = threadIdx.x; k < deg; k += blockDim.x) s.row_eid[b + k] = pb[k];
        }
        if (SUM_HERE) {
            if (threadIdx.x == 0) s.vd[i] = dsqrt(kbn_merge_buf(kb, deg, four_nw(s, i)));
        } else if (inshm) {
            for (int k = threadIdx.x; k < deg; k += blockDim.x) slot[k] = kb[k];
        }
        __syncthreads();
    }
}

template <bool UNIF, bool SUM_HERE>
__global__ void __launch_bounds__(512) k_edge_block(Sweep s, int begin, int end, int cap)
{
    extern __shared__ __align__(16) unsigned char smb[];
    __shared__ int descents;
    if (skipped(s)) return;
    double delta = 0.0;
    for (int j = begin + blockIdx.x; j < end; j += gridDim.x) {
        const long long o = s.ioff[j];
        const int nc = (int)(s.ioff[j + 1] - o);
        double *slot = s.bkey_e + s.bofs_e[j - s.be0];
        const bool inshm = nc <= cap;
        double *kb = inshm ? (double *)smb : slot;
        int2 *pb = inshm ? (int2 *)((double *)smb + cap) : s.scratch_v + (long long)blockIdx.x * s.scratch_stride;
        if (threadIdx.x == 0) descents = 0;
        for (int k = threadIdx.x; k < nc; k += blockDim.x) {
            int2 pr = s.pairs[o + k];
            pb[k] = pr;
            kb[k] = dadd(prod<UNIF>(s, pr.x), prod<UNIF>(s, pr.y));
        }
        __syncthreads();
        int d = 0;
        for (int k = threadIdx.x; k + 1 < nc; k += blockDim.x) d += kb[k + 1] < kb[k];
        if (d) atomicAdd(&descents, d);
        __syncthreads();
        const int nd = descents;
        if (nd) {
            fix_order(kb, pb, nc, threadIdx.x, blockDim.x, BlockSync(), BlockAny(), far_from_sorted(nd, nc));
            for (int k = threadIdx.x; k < nc; k += blockDim.x) s.pairs[o + k] = pb[k];
        }
        if (SUM_HERE) {
            if (threadIdx.x == 0) {
                const int u = s.eu[j], v = s.ev[j];
                delta = fmax(delta, finish_edge<UNIF>(s, j, u, v, kbn_merge_buf(kb, nc, self_term<UNIF>(s, j, u, v))));
            }
        } else if (inshm) {
            for (int k = threadIdx.x; k < nc; k += blockDim.x) slot[k] = kb[k];
        }
        __syncthreads();
    }
    if (SUM_HERE) block_max_to(max_slot(s), delta);
}

// The sequential sums of the block items' sorted slots, in 32-thread
// blocks.  A chain of thousands of terms is bound by the latency of its
// additions, so each BBIG item (the longest) gets a block of its own, one
// lane working, and the block scheduler spreads those over the SMs; the
// BBLOCK items follow, one lane each.  Both ranges are ordered longest first.
template <bool UNIF>
__global__ void __launch_bounds__(32) k_vertex_block_sum(Sweep s, int big0, int nbig, int blk0, int nblk)
{
    extern __shared__ __align__(16) unsigned char smw[];
    if (skipped(s)) return;
    int i;
    if ((int)blockIdx.x < nbig) {
        // a hub row: the whole warp streams its terms
        i = big0 + (int)blockIdx.x;
        const int deg = (int)(s.row_off[i + 1] - s.row_off[i]);
        const double v = kbn_merge_stream_warp(s.bkey_v + s.bofs_v[i - s.bv0], deg, four_nw(s, i), (double *)smw,
                                               (int)threadIdx.x);
        if (threadIdx.x == 0) s.vd[i] = dsqrt(v);
        return;
    } else {
        const int t = ((int)blockIdx.x - nbig) * 32 + (int)threadIdx.x;
        if (t >= nblk) return;
        i = blk0 + t;
    }
    const int deg = (int)(s.row_off[i + 1] - s.row_off[i]);
    s.vd[i] = dsqrt(kbn_merge_stream(s.bkey_v + s.bofs_v[i - s.bv0], deg, four_nw(s, i)));
}

template <bool UNIF>
__global__ void __launch_bounds__(32) k_edge_block_sum(Sweep s, int big0, int nbig, int blk0, int nblk)
{
    extern __shared__ __align__(16) unsigned char smw[];
    if (skipped(s)) return;
    int j = -1;
    if ((int)blockIdx.x >= nbig) {
        const int t = ((int)blockIdx.x - nbig) * 32 + (int)threadIdx.x;
        if (t < nblk) j = blk0 + t;
    }
    double delta = 0.0;
    if ((int)blockIdx.x < nbig) {
        // a hub edge: the whole warp streams its terms
        j = big0 + (int)blockIdx.x;
        const int u = s.eu[j], v = s.ev[j];
        const int nc = (int)(s.ioff[j + 1] - s.ioff[j]);
        const double sum = kbn_merge_stream_warp(s.bkey_e + s.bofs_e[j - s.be0], nc, self_term<UNIF>(s, j, u, v),
                                                 (double *)smw, (int)threadIdx.x);
        if (threadIdx.x == 0) delta = finish_edge<UNIF>(s, j, u, v, sum);
    } else if (j >= 0) {
        const int u = s.eu[j], v = s.ev[j];
        const int nc = (int)(s.ioff[j + 1] - s.ioff[j]);
        delta = finish_edge<UNIF>(s, j, u, v, kbn_merge_stream(s.bkey_e + s.bofs_e[j - s.be0], nc,
                                                               self_term<UNIF>(s, j, u, v)));
    }
    block_max_to(max_slot(s), delta);
}

// ---- launch of one sweep ------------------------------------------------------------

struct Bins {
    int start[NB + 1];
    bool has(int b) const { return start[b + 1] > start[b]; }
    int count(int b) const { return start[b + 1] - start[b]; }
};

inline unsigned grid_for(long long n, int threads, long long cap_blocks)
{
    long long b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > cap_blocks) b = cap_blocks;
    return (unsigned)b;
}

struct LaunchCfg {
    int sms;
    int block_cap;                  // BBIG edges: stored terms in shared memory (16 B each)
    int vblock_cap;                 // BBIG rows: stored terms in shared memory (12 B each)
    cudaStream_t st, side, side2;   // streamed items on st; hubs on side, other block items on side2
    cudaEvent_t fork, join, join2;
    cudaStream_t side3;             // thread-per-item bins beside the streamed items (null: on st)
    cudaEvent_t join3;
};

// Thread bins run as concurrent branches only on graphs up to this many
// edges, where the sweep is bound by launch latency: measured 7-9 % faster
// sweeps from 10K to 120K edges, but 6 % slower on the 28M-edge power-law
// graph, whose large bins then crowd the streamed and block kernels.
constexpr long long BRANCH_MAX_EDGES = 4LL << 20;

constexpr int THR = 128;
constexpr int MED_THR = 256;
// The packed sort uses 10 bytes of shared memory per term (word + low bits).
// The launches ask for 12 (vertices) and 16 (edges), which holds them to 4
// and 3 CTAs per SM: measured on the 28M-edge power-law fit, letting them
// fill the SMs crowds out the block-bin kernels running concurrently on the
// side streams, and the sweep takes 6 % longer.
inline size_t med_smem_vertex() { return (size_t)(MED_THR / 32) * MED_CAP * (8 + 4); }
inline size_t med_smem_edge() { return (size_t)(MED_THR / 32) * MED_CAP * (8 + 8); }

template <bool UNIF>
Status set_sweep_attributes(int block_cap, int vblock_cap)
{
    DRESS_CUDA_TRY(cudaFuncSetAttribute(k_vertex_med_sort<UNIF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)med_smem_vertex()));
    DRESS_CUDA_TRY(cudaFuncSetAttribute(k_edge_med_sort<UNIF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)med_smem_edge()));
    DRESS_CUDA_TRY(cudaFuncSetAttribute(k_vertex_block<UNIF, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        std::max(BIG_CAP, vblock_cap) * 12));
    DRESS_CUDA_TRY(cudaFuncSetAttribute(k_edge_block<UNIF, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        std::max(BIG_CAP, block_cap) * 16));
    return Status::Ok();
}

// Block items on the side stream: the largest (one block per SM, full shared
// memory) first, then the ones up to BIG_CAP terms (several blocks per SM).
template <bool UNIF, bool EDGE>
void launch_blocks(const Sweep &s, const Bins &b, const LaunchCfg &c)
{
    // the hubs' sorts and sums on one stream, so their long chains start as
    // early as possible; the smaller block items beside them on another
    const int nblk = b.count(BBLOCK), nbig = b.count(BBIG);
    if (nbig > 0) {
        if (EDGE) {
            count_launch(), k_edge_block<UNIF, false><<<grid_for(nbig, 1, c.sms), 512, (size_t)c.block_cap * 16,
                                                  c.side>>>(s, b.start[BBIG], b.start[BBIG + 1], c.block_cap);
            count_launch(), k_edge_block_sum<UNIF><<<nbig, 32, HUB_SMEM, c.side>>>(s, b.start[BBIG], nbig, 0, 0);
        } else {
            count_launch(), k_vertex_block<UNIF, false><<<grid_for(nbig, 1, c.sms), 512, (size_t)c.vblock_cap * 12,
                                                    c.side>>>(s, b.start[BBIG], b.start[BBIG + 1], c.vblock_cap);
            count_launch(), k_vertex_block_sum<UNIF><<<nbig, 32, HUB_SMEM, c.side>>>(s, b.start[BBIG], nbig, 0, 0);
        }
    }
    if (nblk > 0) {
        const unsigned g = (unsigned)((nblk + 31) / 32);
        if (EDGE) {
            count_launch(), k_edge_block<UNIF, false><<<grid_for(nblk, 1, 3 * c.sms), 512, (size_t)BIG_CAP * 16,
                                                 c.side2>>>(s, b.start[BBLOCK], b.start[BBLOCK + 1], BIG_CAP);
            count_launch(), k_edge_block_sum<UNIF><<<g, 32, 0, c.side2>>>(s, 0, 0, b.start[BBLOCK], nblk);
        } else {
            count_launch(), k_vertex_block<UNIF, false><<<grid_for(nblk, 1, 4 * c.sms), 512, (size_t)BIG_CAP * 12,
                                                   c.side2>>>(s, b.start[BBLOCK], b.start[BBLOCK + 1], BIG_CAP);
            count_launch(), k_vertex_block_sum<UNIF><<<g, 32, 0, c.side2>>>(s, 0, 0, b.start[BBLOCK], nblk);
        }
    }
}

// Streamed items: one pass over all of them, then the queued ones sorted and finished.
template <bool UNIF, bool EDGE>
void launch_med(const Sweep &s, const Bins &b, const LaunchCfg &c)
{
    if (!b.has(BMED)) return;
    const unsigned g = grid_for(b.count(BMED), MED_THR, 8 * c.sms);
    const unsigned gq = grid_for(b.count(BMED), MED_THR / 32, 8 * c.sms);
    const unsigned gs = grid_for(b.count(BMED), THR, 16 * c.sms);
    if (EDGE) {
        count_launch(), k_edge_med<UNIF><<<g, MED_THR, 0, c.st>>>(s, b.start[BMED], b.start[BMED + 1]);
        count_launch(), k_edge_med_sort<UNIF><<<gq, MED_THR, med_smem_edge(), c.st>>>(s);
        count_launch(), k_edge_med_sum<UNIF><<<gs, THR, 0, c.st>>>(s);
    } else {
        count_launch(), k_vertex_med<UNIF><<<g, MED_THR, 0, c.st>>>(s, b.start[BMED], b.start[BMED + 1]);
        count_launch(), k_vertex_med_sort<UNIF><<<gq, MED_THR, med_smem_vertex(), c.st>>>(s);
        count_launch(), k_vertex_med_sum<UNIF><<<gs, THR, 0, c.st>>>(s);
    }
}

// One sweep: vertex phase, then edge phase.  Within a phase the block items
// run on the side stream, concurrently with everything else on the main
// stream; the phase ends when both are done.
// The thread-per-item bins of a phase, the larger ones first, alternating
// between two streams (the same stream twice keeps them in one queue).
template <bool UNIF, bool EDGE>
void launch_thr(const Sweep &s, const Bins &b, const LaunchCfg &c, cudaStream_t q0, cudaStream_t q1)
{
    const int bins[5] = {B16, B8, B4, B2, B0};
    int k = 0;
    for (int bi : bins) {
        if (!b.has(bi)) continue;
        cudaStream_t q = (k++ & 1) ? q1 : q0;
        const unsigned gr = grid_for(b.count(bi), THR, 16 * c.sms);
        const int lo = b.start[bi], hi = b.start[bi + 1];
        count_launch();
        switch (bi) {
        case B16: EDGE ? k_edge_thr<16, UNIF><<<gr, THR, 0, q>>>(s, lo, hi) : k_vertex_thr<16, UNIF><<<gr, THR, 0, q>>>(s, lo, hi); break;
        case B8: EDGE ? k_edge_thr<8, UNIF><<<gr, THR, 0, q>>>(s, lo, hi) : k_vertex_thr<8, UNIF><<<gr, THR, 0, q>>>(s, lo, hi); break;
        case B4: EDGE ? k_edge_thr<4, UNIF><<<gr, THR, 0, q>>>(s, lo, hi) : k_vertex_thr<4, UNIF><<<gr, THR, 0, q>>>(s, lo, hi); break;
        case B2: EDGE ? k_edge_thr<2, UNIF><<<gr, THR, 0, q>>>(s, lo, hi) : k_vertex_thr<2, UNIF><<<gr, THR, 0, q>>>(s, lo, hi); break;
        default: EDGE ? k_edge_thr<0, UNIF><<<gr, THR, 0, q>>>(s, lo, hi) : k_vertex_thr<0, UNIF><<<gr, THR, 0, q>>>(s, lo, hi); break;
        }
    }
}

// One phase.  The bins are independent of each other, so they run as
// concurrent branches: block items on side (hubs) and side2, the streamed
// items' chain on st, the thread bins on side3 -- or, without streamed
// items, on st and side3 alternately.  Captured into a CUDA graph, the
// branches launch without waiting for one another.
template <bool UNIF, bool EDGE>
Status launch_phase(const Sweep &s, const Bins &b, const LaunchCfg &c)
{
    const bool blocks = b.has(BBLOCK) || b.has(BBIG);
    const bool med = b.has(BMED);
    int nthr = 0;
    for (int bi : {B16, B8, B4, B2, B0}) nthr += b.has(bi);
    const bool split = c.side3 && nthr > 0 && (med || nthr > 1);
    if (blocks || split) DRESS_CUDA_TRY(cudaEventRecord(c.fork, c.st));
    if (blocks) {
        DRESS_CUDA_TRY(cudaStreamWaitEvent(c.side, c.fork, 0));
        DRESS_CUDA_TRY(cudaStreamWaitEvent(c.side2, c.fork, 0));
        launch_blocks<UNIF, EDGE>(s, b, c);
    }
    if (split) {
        DRESS_CUDA_TRY(cudaStreamWaitEvent(c.side3, c.fork, 0));
        if (med) launch_thr<UNIF, EDGE>(s, b, c, c.side3, c.side3);
        else launch_thr<UNIF, EDGE>(s, b, c, c.st, c.side3);
    }
    launch_med<UNIF, EDGE>(s, b, c);
    if (!split) launch_thr<UNIF, EDGE>(s, b, c, c.st, c.st);
    if (blocks) {
        DRESS_CUDA_TRY(cudaEventRecord(c.join, c.side));
        DRESS_CUDA_TRY(cudaEventRecord(c.join2, c.side2));
        DRESS_CUDA_TRY(cudaStreamWaitEvent(c.st, c.join, 0));
        DRESS_CUDA_TRY(cudaStreamWaitEvent(c.st, c.join2, 0));
    }
    if (split) {
        DRESS_CUDA_TRY(cudaEventRecord(c.join3, c.side3));
        DRESS_CUDA_TRY(cudaStreamWaitEvent(c.st, c.join3, 0));
    }
    return Status::Ok();
}

template <bool UNIF>
Status launch_sweep(const Sweep &s, const Bins &vb, const Bins &eb, const LaunchCfg &c)
{
    DRESS_CUDA_TRY(cudaMemsetAsync(s.qcount, 0, 2 * sizeof(unsigned), c.st));
    DRESS_TRY((launch_phase<UNIF, false>(s, vb, c)));
    DRESS_TRY((launch_phase<UNIF, true>(s, eb, c)));
    DRESS_CUDA_TRY(cudaGetLastError());
    return Status::Ok();
}

}  // namespace sweep
}  // namespace dress
