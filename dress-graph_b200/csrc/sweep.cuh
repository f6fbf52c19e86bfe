// sweep.cuh -- the per-sweep kernels of the single-graph fit (fit_graph.cu).
//
// Reference: libdress/src/dress.c:556-591 (vertex norms, edge update) with
// the sorted KBN sum of dress.c:51-66.
//
// Items (vertices, edges) are binned by their number of STORED terms: the
// row's slots for a vertex, the common-neighbour pairs for an edge.  Every
// item has one more term, its self term (4*nw for a vertex, the self/own-edge
// term for an edge).
//
// Every item's terms are streamed once, in storage order, into a certified
// sum (CSum, common.cuh): partial sums per thread, merged across the lanes or
// warps that share the item.  When the certificate holds -- all but about one
// item in a billion -- the value is the reference's sorted-KBN result bit for
// bit.  Otherwise the item is queued, and after the phase one block per
// queued item gathers its terms, sorts them and runs the reference's
// sequential KBN (k_*_exact).  No sweep sorts anything else, and no term
// order is kept between sweeps.
//
//   bins: 0 stored terms; <=2, <=4, <=8, <=16 (one thread per item);
//   <=MED_CAP (a group of 8, 16 or 32 lanes per item); <=BIG_CAP (a warp per
//   item); more (one block per item, largest first).
#pragma once
#include <algorithm>
#include <climits>

#include "common.cuh"
#include "engine.h"

namespace dress {
namespace sweep {

constexpr int NB = 8;
constexpr int MED_CAP = 512;        // stored terms of a warp item
constexpr int BIG_CAP = 4096;       // block items are split here (largest first either way)
enum { B0 = 0, B2, B4, B8, B16, BMED, BBLOCK, BBIG };

__host__ __device__ __forceinline__ int bin_of(long long n)
{
    return n == 0 ? B0 : n <= 2 ? B2 : n <= 4 ? B4 : n <= 8 ? B8 : n <= 16 ? B16 : n <= MED_CAP ? BMED
         : n <= BIG_CAP ? BBLOCK : BBIG;
}

// Fine keys of the renumbering: the coarse bins, with the warp bin split by
// exact term count, longest first -- the longest items start first.
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
    const int *row_eid;            // [S]  slot edge ids
    const int *eu, *ev;            // [E]
    const double *w;               // [E] (weighted graphs)
    double wc;                     // the weight when all are equal
    const double *nw;              // [N], or null when every vertex weight is 1.0
    const long long *ioff;         // [E+1]
    const int2 *pairs;             // [T]  common-neighbour edge pairs
    double *vd;                    // [N]
    unsigned long long *maxd;      // convergence ring
    const double *d, *p;           // current values and products
    double *dn, *pn;               // next values and products
    const int *iter;               // device: index of the sweep being run
    int max_iter;                  // sweeps at or past it return at once
    double eps;
    int *qv, *qe;                  // items whose certificate failed (vertices, edges)
    unsigned *qcount;              // [2] queue lengths, cleared by the exact kernels
    double *scratch;               // exact sorts of items beyond shared memory, per block
    long long scratch_stride;
    int exact_cap;                 // terms an exact-sort block holds in shared memory
    int force_exact;               // queue every item (tests of the exact path)
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

// the edge's own product w*d, from its weight and value (the bits of p[j])
template <bool UNIF>
__device__ __forceinline__ double own_prod(const Sweep &s, int j, double dj)
{
    return dmul(UNIF ? s.wc : s.w[j], dj);
}

// dress.c:456-463: 4nw_u + own (FORWARD/BACKWARD), else 4nw_u + 4nw_v + 2 own
__device__ __forceinline__ double self_term(const Sweep &s, int u, int v, double own)
{
    const double a = four_nw(s, u);
    if (s.fwd) return dadd(a, own);
    return dadd(dadd(a, four_nw(s, v)), dmul(2.0, own));
}

// a pair term: w[eu] d[eu] + w[ev] d[ev] (dress.c:488-489)
template <bool UNIF>
__device__ __forceinline__ double pair_term(const Sweep &s, int2 pr)
{
    return dadd(prod<UNIF>(s, pr.x), prod<UNIF>(s, pr.y));
}

// edge value from its numerator; stores d_next (and p_next), returns |delta|
template <bool UNIF>
__device__ __forceinline__ double finish_edge(const Sweep &s, int j, int u, int v, double dj, double num)
{
    const double den = dmul(s.vd[u], s.vd[v]);
    const double r = den > 0.0 ? ddiv(num, den) : 0.0;
    s.dn[j] = r;
    if (!UNIF) s.pn[j] = dmul(s.w[j], r);
    return fabs(dsub(dj, r));
}

__device__ __forceinline__ void queue_item(int *q, unsigned *count, int item)
{
    q[atomicAdd(count, 1u)] = item;
}

// ---- thread per item --------------------------------------------------------------

// The thread and group kernels wait on dependent gathers (row slot -> value),
// so they ask for RESIDENT blocks of 256 threads per SM (at most 40
// registers): the extra warps hide the loads.  Their grids are one wave of
// RESIDENT blocks per SM, so no SM idles through a partial last wave.
// Measured on the 28M-edge Chung-Lu fit: 1.68 -> 1.50 ms per weighted sweep,
// 1.59 -> 1.44 ms unweighted.
constexpr int RESIDENT = 6;
constexpr int THR = 256;

template <bool UNIF>
__global__ void __launch_bounds__(THR, RESIDENT) k_vertex_thr(Sweep s, int begin, int end)
{
    if (skipped(s)) return;
    for (int i = begin + blockIdx.x * blockDim.x + threadIdx.x; i < end; i += gridDim.x * blockDim.x) {
        const long long rb = s.row_off[i];
        const int deg = (int)(s.row_off[i + 1] - rb);
        const int *re = s.row_eid + rb;
        CSum q;
        q.init();
        q.add(four_nw(s, i));
        int k = 0;
        for (; k + 4 <= deg; k += 4) {
            const int e0 = re[k], e1 = re[k + 1], e2 = re[k + 2], e3 = re[k + 3];
            const double t0 = prod<UNIF>(s, e0), t1 = prod<UNIF>(s, e1);
            const double t2 = prod<UNIF>(s, e2), t3 = prod<UNIF>(s, e3);
            q.add(t0);
            q.add(t1);
            q.add(t2);
            q.add(t3);
        }
        for (; k < deg; ++k) q.add(prod<UNIF>(s, re[k]));
        double sum;
        if (!s.force_exact && q.result(sum)) s.vd[i] = dsqrt(sum);
        else queue_item(s.qv, &s.qcount[0], i);
    }
}

// PAIRS false: the edges without common neighbours (the sum is the self
// term).  Edge kernels take the items [begin, end) of `list` (edge ids), or
// the edge ids [begin, end) themselves when list is null.
template <bool UNIF, bool PAIRS>
__global__ void __launch_bounds__(THR, RESIDENT) k_edge_thr(Sweep s, const int *list, int begin, int end)
{
    if (skipped(s)) return;
    double lmax = 0.0;
    for (int x = begin + blockIdx.x * blockDim.x + threadIdx.x; x < end; x += gridDim.x * blockDim.x) {
        const int j = list ? list[x] : x;
        const int u = s.eu[j], v = s.ev[j];
        const double dj = s.d[j];
        const double self = self_term(s, u, v, own_prod<UNIF>(s, j, dj));
        double num;
        if (PAIRS) {
            const long long pb = s.ioff[j];
            const int n = (int)(s.ioff[j + 1] - pb);
            const int2 *pp = s.pairs + pb;
            CSum q;
            q.init();
            q.add(self);
            int k = 0;
            for (; k + 4 <= n; k += 4) {
                const int2 p0 = pp[k], p1 = pp[k + 1], p2 = pp[k + 2], p3 = pp[k + 3];
                const double t0 = pair_term<UNIF>(s, p0), t1 = pair_term<UNIF>(s, p1);
                const double t2 = pair_term<UNIF>(s, p2), t3 = pair_term<UNIF>(s, p3);
                q.add(t0);
                q.add(t1);
                q.add(t2);
                q.add(t3);
            }
            for (; k < n; ++k) q.add(pair_term<UNIF>(s, pp[k]));
            if (s.force_exact || !q.result(num)) {
                queue_item(s.qe, &s.qcount[1], j);
                continue;
            }
        } else {
            num = dadd(self, 0.0);     // one term: the reference's sum + comp
            if (s.force_exact) {
                queue_item(s.qe, &s.qcount[1], j);
                continue;
            }
        }
        lmax = fmax(lmax, finish_edge<UNIF>(s, j, u, v, dj, num));
    }
    block_max_to(max_slot(s), lmax);
}

// ---- a group of GW lanes per item ------------------------------------------------------
// The warp bin (17..MED_CAP terms) is split by term count into groups of 8,
// 16 or 32 lanes per item (at most 8 or 16 terms a lane in the smaller
// ones): fewer idle lanes and merge rounds for short items.  A warp takes
// 32 / GW consecutive items per step, so the loop control and the lane
// merge stay warp-uniform.

constexpr int WARP_THR = 256;

template <bool UNIF, int GW>
__global__ void __launch_bounds__(WARP_THR, RESIDENT) k_vertex_grp(Sweep s, int begin, int end)
{
    if (skipped(s)) return;
    constexpr int IPW = 32 / GW;                  // items per warp step
    const int lane = threadIdx.x & (GW - 1);
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int i0 = begin + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * IPW; i0 < end; i0 += nwarps * IPW) {
        const int i = i0 + (int)((threadIdx.x & 31) / GW);
        const bool valid = i < end;
        long long rb = 0;
        int deg = 0;
        if (valid) {
            rb = s.row_off[i];
            deg = (int)(s.row_off[i + 1] - rb);
        }
        const int *re = s.row_eid + rb;
        CSum q;
        q.init();
        if (valid && lane == 0) q.add(four_nw(s, i));
        int k = lane;
        for (; k + 3 * GW < deg; k += 4 * GW) {
            const int e0 = re[k], e1 = re[k + GW], e2 = re[k + 2 * GW], e3 = re[k + 3 * GW];
            const double t0 = prod<UNIF>(s, e0), t1 = prod<UNIF>(s, e1);
            const double t2 = prod<UNIF>(s, e2), t3 = prod<UNIF>(s, e3);
            q.add(t0);
            q.add(t1);
            q.add(t2);
            q.add(t3);
        }
        for (; k < deg; k += GW) q.add(prod<UNIF>(s, re[k]));
        q.merge_lanes(GW);
        if (valid && lane == 0) {
            double sum;
            if (!s.force_exact && q.result(sum)) s.vd[i] = dsqrt(sum);
            else queue_item(s.qv, &s.qcount[0], i);
        }
    }
}

template <bool UNIF, int GW>
__global__ void __launch_bounds__(WARP_THR, RESIDENT) k_edge_grp(Sweep s, const int *list, int begin, int end)
{
    if (skipped(s)) return;
    constexpr int IPW = 32 / GW;
    const int lane = threadIdx.x & (GW - 1);
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    double lmax = 0.0;
    for (int x0 = begin + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * IPW; x0 < end; x0 += nwarps * IPW) {
        const int x = x0 + (int)((threadIdx.x & 31) / GW);
        const bool valid = x < end;
        const int j = valid ? (list ? list[x] : x) : 0;
        long long pb = 0;
        int n = 0;
        if (valid) {
            pb = s.ioff[j];
            n = (int)(s.ioff[j + 1] - pb);
        }
        const int2 *pp = s.pairs + pb;
        int u = 0, v = 0;
        double dj = 0.0;
        CSum q;
        q.init();
        if (valid && lane == 0) {
            u = s.eu[j];
            v = s.ev[j];
            dj = s.d[j];
            q.add(self_term(s, u, v, own_prod<UNIF>(s, j, dj)));
        }
        int k = lane;
        for (; k + 3 * GW < n; k += 4 * GW) {
            const int2 p0 = pp[k], p1 = pp[k + GW], p2 = pp[k + 2 * GW], p3 = pp[k + 3 * GW];
            const double t0 = pair_term<UNIF>(s, p0), t1 = pair_term<UNIF>(s, p1);
            const double t2 = pair_term<UNIF>(s, p2), t3 = pair_term<UNIF>(s, p3);
            q.add(t0);
            q.add(t1);
            q.add(t2);
            q.add(t3);
        }
        for (; k < n; k += GW) q.add(pair_term<UNIF>(s, pp[k]));
        q.merge_lanes(GW);
        if (valid && lane == 0) {
            double num;
            if (!s.force_exact && q.result(num)) lmax = fmax(lmax, finish_edge<UNIF>(s, j, u, v, dj, num));
            else queue_item(s.qe, &s.qcount[1], j);
        }
    }
    block_max_to(max_slot(s), lmax);
}

// ---- one block per item ----------------------------------------------------------------

constexpr int BLK_THR = 512;

// merge of the block's per-warp sums into thread 0 (every thread calls it)
__device__ __forceinline__ void merge_block(CSum &q)
{
    __shared__ double ps[BLK_THR / 32], pc[BLK_THR / 32], pa[BLK_THR / 32], pm[BLK_THR / 32];
    __shared__ int pn[BLK_THR / 32];
    q.merge_lanes(32);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        ps[wid] = q.s;
        pc[wid] = q.c;
        pa[wid] = q.a;
        pm[wid] = q.m;
        pn[wid] = q.n;
    }
    __syncthreads();
    if (threadIdx.x == 0)
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) q.merge(ps[w], pc[w], pa[w], pm[w], pn[w]);
    __syncthreads();
}

template <bool UNIF>
__global__ void __launch_bounds__(BLK_THR) k_vertex_blk(Sweep s, int begin, int end)
{
    if (skipped(s)) return;
    for (int i = begin + (int)blockIdx.x; i < end; i += gridDim.x) {
        const long long rb = s.row_off[i];
        const int deg = (int)(s.row_off[i + 1] - rb);
        const int *re = s.row_eid + rb;
        CSum q;
        q.init();
        if (threadIdx.x == 0) q.add(four_nw(s, i));
        int k = threadIdx.x;
        for (; k + 3 * BLK_THR < deg; k += 4 * BLK_THR) {
            const int e0 = re[k], e1 = re[k + BLK_THR], e2 = re[k + 2 * BLK_THR], e3 = re[k + 3 * BLK_THR];
            const double t0 = prod<UNIF>(s, e0), t1 = prod<UNIF>(s, e1);
            const double t2 = prod<UNIF>(s, e2), t3 = prod<UNIF>(s, e3);
            q.add(t0);
            q.add(t1);
            q.add(t2);
            q.add(t3);
        }
        for (; k < deg; k += BLK_THR) q.add(prod<UNIF>(s, re[k]));
        merge_block(q);
        if (threadIdx.x == 0) {
            double sum;
            if (!s.force_exact && q.result(sum)) s.vd[i] = dsqrt(sum);
            else queue_item(s.qv, &s.qcount[0], i);
        }
    }
}

template <bool UNIF>
__global__ void __launch_bounds__(BLK_THR) k_edge_blk(Sweep s, const int *list, int begin, int end)
{
    if (skipped(s)) return;
    double lmax = 0.0;
    for (int x = begin + (int)blockIdx.x; x < end; x += gridDim.x) {
        const int j = list ? list[x] : x;
        const long long pb = s.ioff[j];
        const int n = (int)(s.ioff[j + 1] - pb);
        const int2 *pp = s.pairs + pb;
        int u = 0, v = 0;
        double dj = 0.0;
        CSum q;
        q.init();
        if (threadIdx.x == 0) {
            u = s.eu[j];
            v = s.ev[j];
            dj = s.d[j];
            q.add(self_term(s, u, v, own_prod<UNIF>(s, j, dj)));
        }
        int k = threadIdx.x;
        for (; k + 3 * BLK_THR < n; k += 4 * BLK_THR) {
            const int2 p0 = pp[k], p1 = pp[k + BLK_THR], p2 = pp[k + 2 * BLK_THR], p3 = pp[k + 3 * BLK_THR];
            const double t0 = pair_term<UNIF>(s, p0), t1 = pair_term<UNIF>(s, p1);
            const double t2 = pair_term<UNIF>(s, p2), t3 = pair_term<UNIF>(s, p3);
            q.add(t0);
            q.add(t1);
            q.add(t2);
            q.add(t3);
        }
        for (; k < n; k += BLK_THR) q.add(pair_term<UNIF>(s, pp[k]));
        merge_block(q);
        if (threadIdx.x == 0) {
            double num;
            if (!s.force_exact && q.result(num)) lmax = fmax(lmax, finish_edge<UNIF>(s, j, u, v, dj, num));
            else queue_item(s.qe, &s.qcount[1], j);
        }
    }
    block_max_to(max_slot(s), lmax);
}

// ---- exact sums of the queued items -------------------------------------------------------
// One block per queued item: the terms are gathered into shared memory (or
// the block's global scratch when they do not fit), sorted ascending, and
// thread 0 runs the reference's sequential KBN over them.  The queue is
// empty in nearly every sweep, and these kernels then return at once.

constexpr int EXACT_THR = 512;

struct BlockBarrier {
    __device__ __forceinline__ void operator()() const { __syncthreads(); }
};

template <bool UNIF>
__global__ void __launch_bounds__(EXACT_THR) k_vertex_exact(Sweep s)
{
    extern __shared__ __align__(16) double keys[];
    if (skipped(s)) return;
    const unsigned cnt = *(volatile unsigned *)&s.qcount[0];
    for (unsigned qi = blockIdx.x; qi < cnt; qi += gridDim.x) {
        const int i = s.qv[qi];
        const long long rb = s.row_off[i];
        const int deg = (int)(s.row_off[i + 1] - rb);
        const int n = deg + 1;
        double *buf = n <= s.exact_cap ? keys : s.scratch + (long long)blockIdx.x * s.scratch_stride;
        for (int k = threadIdx.x; k < deg; k += blockDim.x) buf[k] = prod<UNIF>(s, s.row_eid[rb + k]);
        if (threadIdx.x == 0) buf[deg] = four_nw(s, i);
        __syncthreads();
        sort_shared(buf, n, (int)threadIdx.x, (int)blockDim.x, BlockBarrier{});
        if (threadIdx.x == 0) s.vd[i] = dsqrt(kbn_sorted_buf(buf, n));
        __syncthreads();
    }
}

template <bool UNIF>
__global__ void __launch_bounds__(EXACT_THR) k_edge_exact(Sweep s)
{
    extern __shared__ __align__(16) double keys[];
    if (skipped(s)) return;
    const unsigned cnt = *(volatile unsigned *)&s.qcount[1];
    double lmax = 0.0;
    for (unsigned qi = blockIdx.x; qi < cnt; qi += gridDim.x) {
        const int j = s.qe[qi];
        const long long pb = s.ioff[j];
        const int np = (int)(s.ioff[j + 1] - pb);
        const int n = np + 1;
        double *buf = n <= s.exact_cap ? keys : s.scratch + (long long)blockIdx.x * s.scratch_stride;
        for (int k = threadIdx.x; k < np; k += blockDim.x) buf[k] = pair_term<UNIF>(s, s.pairs[pb + k]);
        const int u = s.eu[j], v = s.ev[j];
        const double dj = s.d[j];
        if (threadIdx.x == 0) buf[np] = self_term(s, u, v, own_prod<UNIF>(s, j, dj));
        __syncthreads();
        sort_shared(buf, n, (int)threadIdx.x, (int)blockDim.x, BlockBarrier{});
        if (threadIdx.x == 0) lmax = fmax(lmax, finish_edge<UNIF>(s, j, u, v, dj, kbn_sorted_buf(buf, n)));
        __syncthreads();
    }
    block_max_to(max_slot(s), lmax);
}

// both queues emptied for the next sweep (after both exact kernels)
__global__ void k_clear_queues(unsigned *qcount)
{
    qcount[0] = 0u;
    qcount[1] = 0u;
}

// ---- launch of one sweep ------------------------------------------------------------

struct Bins {
    int start[NB + 1];
    int med[4];                    // the warp bin split by term count (see launch_phase)
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
    int exact_grid;                 // blocks of the exact-sum kernels
    size_t exact_smem;              // their shared memory (exact_cap doubles)
    cudaStream_t st, side;          // block items run on side, concurrently with the rest
    cudaEvent_t fork, join;
};

template <bool UNIF>
Status set_sweep_attributes(size_t exact_smem)
{
    DRESS_CUDA_TRY(cudaFuncSetAttribute(k_vertex_exact<UNIF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)exact_smem));
    DRESS_CUDA_TRY(cudaFuncSetAttribute(k_edge_exact<UNIF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)exact_smem));
    return Status::Ok();
}

// The edge items of a sweep: the edges without common neighbours are the
// ids [0, e0); the others are listed by size class in `list`:
// [cls[0], cls[1]) 1..16 pairs (a thread each), [cls[1], cls[2]) 257..512,
// [cls[2], cls[3]) 65..256, [cls[3], cls[4]) 17..64 (lane groups of 32, 16,
// 8), [cls[4], cls[5]) 513..BIG_CAP (a warp each), [cls[5], cls[6]) more (a
// block each).
struct EdgeClasses {
    int e0;
    const int *list;
    int cls[7];
};

template <bool UNIF>
void launch_grp(const Sweep &s, const int *list, int lo, int hi, int gw, const LaunchCfg &c, bool edge)
{
    if (hi <= lo) return;
    const unsigned g = grid_for((long long)(hi - lo) * gw, WARP_THR, (long long)RESIDENT * c.sms);
    count_launch();
    switch (gw) {
    case 32: edge ? k_edge_grp<UNIF, 32><<<g, WARP_THR, 0, c.st>>>(s, list, lo, hi)
                  : k_vertex_grp<UNIF, 32><<<g, WARP_THR, 0, c.st>>>(s, lo, hi); break;
    case 16: edge ? k_edge_grp<UNIF, 16><<<g, WARP_THR, 0, c.st>>>(s, list, lo, hi)
                  : k_vertex_grp<UNIF, 16><<<g, WARP_THR, 0, c.st>>>(s, lo, hi); break;
    default: edge ? k_edge_grp<UNIF, 8><<<g, WARP_THR, 0, c.st>>>(s, list, lo, hi)
                  : k_vertex_grp<UNIF, 8><<<g, WARP_THR, 0, c.st>>>(s, lo, hi); break;
    }
}

// Vertex phase: rows beyond BIG_CAP slots a block each on the side stream,
// beside the warp and thread rows on the main stream; then the exact sums
// of the queued rows.
template <bool UNIF>
Status launch_vertex_phase(const Sweep &s, const Bins &b, const LaunchCfg &c)
{
    const bool blocks = b.has(BBIG);
    if (blocks) {
        DRESS_CUDA_TRY(cudaEventRecord(c.fork, c.st));
        DRESS_CUDA_TRY(cudaStreamWaitEvent(c.side, c.fork, 0));
        const int lo = b.start[BBIG], hi = b.start[BBIG + 1];
        count_launch(), k_vertex_blk<UNIF><<<grid_for(hi - lo, 1, 8LL * c.sms), BLK_THR, 0, c.side>>>(s, lo, hi);
    }
    launch_grp<UNIF>(s, nullptr, b.start[BBLOCK], b.start[BBLOCK + 1], 32, c, false);
    if (b.has(BMED)) {
        launch_grp<UNIF>(s, nullptr, b.med[0], b.med[1], 32, c, false);
        launch_grp<UNIF>(s, nullptr, b.med[1], b.med[2], 16, c, false);
        launch_grp<UNIF>(s, nullptr, b.med[2], b.med[3], 8, c, false);
    }
    {
        const int lo = b.start[B0], hi = b.start[BMED];
        if (hi > lo)
            count_launch(), k_vertex_thr<UNIF><<<grid_for(hi - lo, THR, (long long)RESIDENT * c.sms), THR, 0, c.st>>>(s, lo, hi);
    }
    if (blocks) {
        DRESS_CUDA_TRY(cudaEventRecord(c.join, c.side));
        DRESS_CUDA_TRY(cudaStreamWaitEvent(c.st, c.join, 0));
    }
    count_launch(), k_vertex_exact<UNIF><<<c.exact_grid, EXACT_THR, c.exact_smem, c.st>>>(s);
    return Status::Ok();
}

// Edge phase: the same shape over the edge classes.
template <bool UNIF>
Status launch_edge_phase(const Sweep &s, const EdgeClasses &ec, const LaunchCfg &c)
{
    const int *L = ec.list;
    const int *k = ec.cls;
    const bool blocks = k[6] > k[5];
    if (blocks) {
        DRESS_CUDA_TRY(cudaEventRecord(c.fork, c.st));
        DRESS_CUDA_TRY(cudaStreamWaitEvent(c.side, c.fork, 0));
        count_launch(), k_edge_blk<UNIF><<<grid_for(k[6] - k[5], 1, 8LL * c.sms), BLK_THR, 0, c.side>>>(
            s, L, k[5], k[6]);
    }
    launch_grp<UNIF>(s, L, k[4], k[5], 32, c, true);
    launch_grp<UNIF>(s, L, k[1], k[2], 32, c, true);
    launch_grp<UNIF>(s, L, k[2], k[3], 16, c, true);
    launch_grp<UNIF>(s, L, k[3], k[4], 8, c, true);
    if (ec.e0 > 0)
        count_launch(), k_edge_thr<UNIF, false><<<grid_for(ec.e0, THR, (long long)RESIDENT * c.sms), THR, 0, c.st>>>(
            s, nullptr, 0, ec.e0);
    if (k[1] > k[0])
        count_launch(), k_edge_thr<UNIF, true><<<grid_for(k[1] - k[0], THR, (long long)RESIDENT * c.sms), THR, 0, c.st>>>(
            s, L, k[0], k[1]);
    if (blocks) {
        DRESS_CUDA_TRY(cudaEventRecord(c.join, c.side));
        DRESS_CUDA_TRY(cudaStreamWaitEvent(c.st, c.join, 0));
    }
    count_launch(), k_edge_exact<UNIF><<<c.exact_grid, EXACT_THR, c.exact_smem, c.st>>>(s);
    return Status::Ok();
}

template <bool UNIF>
Status launch_sweep(const Sweep &s, const Bins &vb, const EdgeClasses &ec, const LaunchCfg &c)
{
    DRESS_TRY(launch_vertex_phase<UNIF>(s, vb, c));
    DRESS_TRY(launch_edge_phase<UNIF>(s, ec, c));
    count_launch(), k_clear_queues<<<1, 1, 0, c.st>>>(s.qcount);
    DRESS_CUDA_TRY(cudaGetLastError());
    return Status::Ok();
}

}  // namespace sweep
}  // namespace dress
