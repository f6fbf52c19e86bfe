// batch.cu -- one persistent launch fits many small subgraphs.
//
// Reference behaviour: the Delta^k / Nabla^k drivers
// (libdress/src/delta_dress_impl.c:171-318, nabla_dress_impl.c:142-311)
// rebuild a CSR per subgraph on the host and call the fit
// (libdress/src/dress.c:546-608) once per subgraph.  Here:
//   * a CTA grabs a chunk of subgraphs of one parent graph from a global
//     counter, copies the parent's packed arrays (edge endpoints, variant
//     weights, CSR rows, common-neighbour pairs) into shared memory once, and
//     its thread groups (one group per subgraph) pull subgraphs from the chunk;
//   * a subgraph is the parent plus a mask: Delta deletes the k vertices of
//     the combination with lexicographic rank s, Nabla gives the k vertices of
//     the ordered tuple with rank s the marker weights sqrt(prime_i); both are
//     unranked in the kernel.  Masking keeps every surviving row's order and
//     every term's value, and the sorted-KBN sums do not depend on the order of
//     their terms, so the values are bit-identical to the rebuilt subgraph's;
//   * each group iterates its subgraph to its own convergence (state d, d_next,
//     vertex norms in shared memory) and appends the live edges' values to the
//     request's value segment (the histogram is built afterwards, hist.cu).
#include <cooperative_groups.h>

#include <map>
#include <mutex>
#include <tuple>

#include "batch.h"
#include "common.cuh"

namespace cg = cooperative_groups;

namespace dress {
namespace {

// The exact sorted KBN of the self term (index cnt) and the live stored
// terms, visited in ascending (value, index) order by repeated scans: no
// storage, O(cnt^2) term evaluations.  Equal values are interchangeable in
// the sum, so this is the reference's "sort, then KBN" (dress.c:51-66).  It
// runs only for the items whose certified sum fails (about one in 1e9).
template <class Terms>
__device__ __noinline__ double sorted_sum_select(double self, int cnt, Terms term)
{
    double pv = -DRESS_INF, s = 0.0, c = 0.0;
    int pj = -1;
    bool first = true;
    for (;;) {
        double bv = DRESS_INF;
        int bj = INT_MAX;
        for (int j = 0; j <= cnt; ++j) {
            double t = self;
            if (j < cnt && !term(j, t)) continue;
            const bool after = t > pv || (t == pv && j > pj);
            const bool better = t < bv || (t == bv && j < bj);
            if (after && better) {
                bv = t;
                bj = j;
            }
        }
        if (bj == INT_MAX) break;
        if (first) {
            s = bv;
            first = false;
        } else {
            kbn_step(s, c, bv);
        }
        pv = bv;
        pj = bj;
    }
    return dadd(s, c);
}

// Sum of the self term and the live ones among cnt stored terms (term(j, t)
// yields stored term j and whether it is alive): a certified sum in stored
// order (CSum, common.cuh), the exact sorted sum where the certificate fails.
template <class Terms>
__device__ __forceinline__ double item_sum(double self, int cnt, const Terms &term, bool force_exact)
{
    if (cnt == 0) return dadd(self, 0.0);        // one term: the reference's sum + comp
    if (force_exact) return sorted_sum_select(self, cnt, term);
    CSum q;
    q.init();
    q.add(self);
    for (int j = 0; j < cnt; ++j) {
        double t;
        if (term(j, t)) q.add(t);
    }
    double r;
    if (q.result(r)) return r;
    return sorted_sum_select(self, cnt, term);
}

__device__ __forceinline__ long long binom_d(int n, int k)
{
    if (k < 0 || k > n) return 0;
    if (k > n - k) k = n - k;
    long long r = 1;
    for (int i = 0; i < k; ++i) r = r * (n - i) / (i + 1);
    return r;
}

__device__ __forceinline__ long long perm_d(int n, int k)
{
    if (k < 0 || k > n) return 0;
    long long r = 1;
    for (int i = 0; i < k; ++i) r *= (n - i);
    return r;
}

__constant__ int c_primes[16] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53};

// sqrt of the (i+1)-th prime for i < 16, sqrt(2i+3) beyond
// (libdress/src/nabla_dress_impl.c:33-46)
__device__ __forceinline__ double marker_weight(int i)
{
    return dsqrt((double)(i < 16 ? c_primes[i] : 2 * i + 3));
}

struct View {
    const int *U, *V, *row_off, *row_eid, *ioff;
    const double *w, *nw, *dinit;
    const int2 *pairs;
};

struct Group {
    int gid, t, size;
    __device__ __forceinline__ void sync() const
    {
        if (size == 32) __syncwarp();
        else asm volatile("bar.sync %0, %1;" ::"r"(gid + 1), "r"(size) : "memory");
    }
    // after group_max: a group wider than a warp has just passed a barrier
    // there; a warp's shuffles order no shared-memory writes
    __device__ __forceinline__ void sync_after_reduce() const
    {
        if (size == 32) __syncwarp();
    }
};

// The masked subgraph of one item: deleted (Delta) or marked (Nabla) vertices.
struct Mask {
    int kind, k;
    const int *v;            // k vertices (shared memory)
    __device__ __forceinline__ bool alive(int x) const
    {
        if (kind != ITEM_DELTA) return true;
        for (int i = 0; i < k; ++i)
            if (v[i] == x) return false;
        return true;
    }
    __device__ __forceinline__ double weight(int x, const double *nw) const
    {
        if (kind == ITEM_PLAIN) return nw ? nw[x] : 1.0;
        if (kind == ITEM_NABLA)
            for (int i = 0; i < k; ++i)
                if (v[i] == x) return marker_weight(i);
        return 1.0;
    }
};

// group-wide sum (int) and max (double); `red` holds 2 x warps-per-group slots
__device__ __forceinline__ double group_max(const Group &g, double v, double *red, int parity)
{
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (g.size == 32) return v;
    int nw = g.size >> 5;
    double *r = red + parity * nw;
    if ((g.t & 31) == 0) r[g.t >> 5] = v;
    g.sync();
    double m = 0.0;
    for (int i = 0; i < nw; ++i) m = fmax(m, r[i]);
    return m;
}

__device__ __forceinline__ int group_sum(const Group &g, int v, double *red, int parity)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (g.size == 32) return v;
    int nw = g.size >> 5;
    double *r = red + parity * nw;
    if ((g.t & 31) == 0) r[g.t >> 5] = (double)v;
    g.sync();
    double s = 0.0;
    for (int i = 0; i < nw; ++i) s += r[i];
    return (int)s;
}

// ---- a whole graph over a thread-block cluster ---------------------------------
// Every thread of the cluster is one member of the group; the state arrays are
// distributed over the CTAs' shared memory, each CTA holding the elements its
// own threads update in the group loops (element i, visited by group thread
// i mod size, lives in CTA (i / B) mod n at ((i / (B n)) B + i mod B), B the
// CTA's threads, n the CTAs).  Other elements are read through distributed
// shared memory.  sync() is the cluster barrier, which also orders the
// shared-memory writes of every CTA (no thread spins).
struct ClusterGroup {
    int t, size;
    double *wsl;                 // this CTA's per-warp reduction slots, two parities
    double *const *part;         // every CTA's two partial slots
    int ncta;
    __device__ __forceinline__ void sync() const { cg::this_cluster().sync(); }
    // after group_max: every thread has just passed its cluster barrier
    __device__ __forceinline__ void sync_after_reduce() const {}
};

struct DArr {
    double *const *tab;          // every CTA's slice (generic addresses)
    int lb, lnc;                 // log2 of the CTA's threads and of the CTAs
    __device__ __forceinline__ double &operator[](int i) const
    {
        const int r = (i >> lb) & ((1 << lnc) - 1);
        const int l = ((i >> (lb + lnc)) << lb) | (i & ((1 << lb) - 1));
        return tab[r][l];
    }
};

template <class Op>
__device__ __forceinline__ double cluster_reduce(const ClusterGroup &g, double v, int parity, Op op)
{
    for (int o = 16; o > 0; o >>= 1) v = op(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int nw = (int)blockDim.x >> 5;
    if ((threadIdx.x & 31) == 0) g.wsl[parity * nw + (threadIdx.x >> 5)] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = g.wsl[parity * nw];
        for (int i = 1; i < nw; ++i) m = op(m, g.wsl[parity * nw + i]);
        g.part[cg::this_cluster().block_rank()][parity] = m;
    }
    g.sync();
    double m = g.part[0][parity];
    for (int r = 1; r < g.ncta; ++r) m = op(m, g.part[r][parity]);
    return m;
}

__device__ __forceinline__ double group_max(const ClusterGroup &g, double v, double *, int parity)
{
    return fmax(0.0, cluster_reduce(g, v, parity, [](double a, double b) { return fmax(a, b); }));
}

__device__ __forceinline__ int group_sum(const ClusterGroup &g, int v, double *, int parity)
{
    return (int)cluster_reduce(g, (double)v, parity, [](double a, double b) { return a + b; });
}

// Stored terms of vertex u's row, w[e] d[e] of every live slot edge
// (dress.c:566-569).  eb (nullable): E bits of group memory, set for the live
// edges of a Delta subgraph; with them a term's liveness is one bit instead
// of its endpoints' lookup against the deleted vertices.
template <class Arr>
struct RowTerms {
    const int *row_eid, *U, *V;
    const double *w;
    Mask mk;
    Arr d0;
    const unsigned *eb;
    int rb, u;
    bool delta;
    __device__ __forceinline__ bool operator()(int j, double &t) const
    {
        const int e = row_eid[rb + j];
        if (delta && !(eb ? ((eb[e >> 5] >> (e & 31)) & 1u) != 0 : mk.alive(U[e] + V[e] - u))) return false;
        t = dmul(w[e], d0[e]);
        return true;
    }
};

// Common-neighbour terms of edge (u, v): w[eu] d[eu] + w[ev] d[ev] of every
// pair whose (u, x) edge is live (dress.c:485-490)
template <class Arr>
struct PairTerms {
    const int2 *pairs;
    const int *U, *V;
    const double *w;
    Mask mk;
    Arr d0;
    const unsigned *eb;
    int pb, u;
    bool delta;
    __device__ __forceinline__ bool operator()(int j, double &t) const
    {
        const int2 pr = pairs[pb + j];
        if (delta && !(eb ? ((eb[pr.x >> 5] >> (pr.x & 31)) & 1u) != 0 : mk.alive(U[pr.x] + V[pr.x] - u)))
            return false;
        t = dadd(dmul(w[pr.x], d0[pr.x]), dmul(w[pr.y], d0[pr.y]));
        return true;
    }
};

template <class Grp, class Arr>
__device__ void fit_item(const ParentDesc &P, const View &G, long long item,
                         const Grp &g, Arr d0, Arr d1, Arr vd, double *red, int *ks,
                         unsigned long long *slot, unsigned *eb)
{
    const int N = P.N, E = P.E;
    const long long s = P.ranks ? P.ranks[item] : P.offset + item * P.stride;
    // ---- unrank the subset / tuple --------------------------------------
    if (g.t == 0 && P.kind != ITEM_PLAIN) {
        long long r = s;
        if (P.kind == ITEM_DELTA) {
            int c = 0;
            for (int i = 0; i < P.k; ++i) {
                for (;;) {
                    long long cnt = binom_d(N - c - 1, P.k - i - 1);
                    if (r < cnt) break;
                    r -= cnt;
                    ++c;
                }
                ks[i] = c++;
            }
        } else {
            for (int i = 0; i < P.k; ++i) {
                long long per = perm_d(N - i - 1, P.k - i - 1);
                long long idx = r / per;
                r -= idx * per;
                int v = 0, seen = -1;
                for (;; ++v) {
                    bool used = false;
                    for (int j = 0; j < i; ++j) used |= ks[j] == v;
                    if (!used && ++seen == idx) break;
                }
                ks[i] = v;
            }
        }
    }
    g.sync();
    Mask mk{P.kind, P.kind == ITEM_PLAIN ? 0 : P.k, ks};

    // ---- live edges, initial values -----------------------------------------
    // a warp's lanes take 32 consecutive edges, so a ballot is a word of bits
    const bool bits = eb && P.kind == ITEM_DELTA;
    int live = 0;
    for (int b0 = g.t & ~31; b0 < E; b0 += g.size) {
        const int e = b0 + (g.t & 31);
        const bool al = e < E && mk.alive(G.U[e]) && mk.alive(G.V[e]);
        if (e < E) d0[e] = P.has_dinit ? G.dinit[e] : 1.0;
        const unsigned word = __ballot_sync(0xffffffffu, al);
        if (bits && (g.t & 31) == 0) eb[b0 >> 5] = word;
        live += al;
    }
    g.sync();                                    // the bits and initial values, group-wide
    live = group_sum(g, live, red, 0);
    if (live == 0 && P.kind != ITEM_PLAIN) {   // the reference skips edgeless subgraphs
        g.sync();
        return;
    }

    // ---- sweeps ------------------------------------------------------------------
    int it = 0;
    double last = 0.0;
    for (; it < P.max_iter; ++it) {
        for (int u = g.t; u < N; u += g.size) {
            if (!mk.alive(u)) continue;
            const int rb = G.row_off[u], deg = G.row_off[u + 1] - rb;
            const RowTerms<Arr> rt{G.row_eid, G.U, G.V, G.w, mk, d0, bits ? eb : nullptr, rb, u, P.kind == ITEM_DELTA};
            vd[u] = dsqrt(item_sum(dmul(4.0, mk.weight(u, G.nw)), deg, rt, P.force_exact != 0));
        }
        g.sync();
        double lmax = 0.0;
        for (int e = g.t; e < E; e += g.size) {
            const int u = G.U[e], v = G.V[e];
            if (P.kind == ITEM_DELTA && !(bits ? ((eb[e >> 5] >> (e & 31)) & 1u) != 0 : mk.alive(u) && mk.alive(v)))
                continue;
            const double own = dmul(G.w[e], d0[e]);
            const double a4u = dmul(4.0, mk.weight(u, G.nw));
            const double self = P.fwd ? dadd(a4u, own) : dadd(dadd(a4u, dmul(4.0, mk.weight(v, G.nw))), dmul(2.0, own));
            const int pb = G.ioff[e], np = G.ioff[e + 1] - pb;
            const PairTerms<Arr> pt{G.pairs, G.U, G.V, G.w, mk, d0, bits ? eb : nullptr, pb, u, P.kind == ITEM_DELTA};
            const double num = item_sum(self, np, pt, P.force_exact != 0);
            const double den = dmul(vd[u], vd[v]);
            const double r = den > 0.0 ? ddiv(num, den) : 0.0;
            d1[e] = r;
            const double dd = fabs(dsub(d0[e], r));
            if (dd > lmax) lmax = dd;
        }
        const double m = group_max(g, lmax, red, (it & 1));
        last = m;
        const Arr t = d0;
        d0 = d1;
        d1 = t;
        // The reduction's barrier already orders this sweep's writes of d1
        // and its reads of vd and d0 before the next sweep's writes; its
        // slots alternate by parity.
        g.sync_after_reduce();
        if (m < P.eps) break;
    }
    const int sweeps = it < P.max_iter ? it + 1 : P.max_iter;

    // ---- plain fit: the final state in edge / vertex order -------------------------
    if (P.kind == ITEM_PLAIN) {
        for (int e = g.t; e < E; e += g.size) P.values[e] = d0[e];
        if (P.max_iter > 0)     // the norms of the last sweep (none without sweeps)
            for (int u = g.t; u < N; u += g.size) P.values[E + u] = vd[u];
        if (g.t == 0) {
            unsigned long long *st = P.stats;
            const int done = P.max_iter > 0 ? sweeps : 0;
            st[ST_SWEEPS] = (unsigned long long)done;
            st[ST_EDGE_ITERS] = (unsigned long long)E * (unsigned long long)done;
            st[ST_FITS] = 1ULL;
            st[ST_ITERATIONS] = (unsigned long long)(it < P.max_iter ? it : P.max_iter);
            st[ST_DELTA] = (unsigned long long)__double_as_longlong(last);
        }
        g.sync();
        return;
    }

    // ---- emit the live values -------------------------------------------------------
    if (g.t == 0) {
        slot[0] = atomicAdd(&P.stats[ST_CURSOR], (unsigned long long)live);
        slot[1] = 0;
        atomicAdd(&P.stats[ST_SWEEPS], (unsigned long long)sweeps);
        atomicAdd(&P.stats[ST_EDGE_ITERS], (unsigned long long)live * (unsigned long long)sweeps);
        atomicAdd(&P.stats[ST_FITS], 1ULL);
    }
    g.sync();
    double *out = P.values + (long long)slot[0];
    double *row = P.multisets ? P.multisets + s * (long long)E : nullptr;
    for (int e = g.t; e < E; e += g.size) {
        bool al = mk.alive(G.U[e]) && mk.alive(G.V[e]);
        if (al) {
            unsigned long long q = atomicAdd(&slot[1], 1ULL);
            out[q] = d0[e];
        }
        if (row) row[e] = al ? d0[e] : __longlong_as_double(0x7ff8000000000000LL);
    }
    g.sync();
}

__host__ __device__ inline long long group_bytes(const BatchLaunch &L)
{
    long long b = 8LL * (2LL * L.maxE + L.maxN) + 8LL * 2 * (L.gsize / 32) + 4LL * (L.maxk > 0 ? L.maxk : 1) + 16 +
                  4LL * ((L.maxE + 31) / 32);       // live-edge bits
    return pl_align(b);
}

__device__ __forceinline__ View view_of(const unsigned char *b, const ParentLayout &PL, const ParentDesc &P)
{
    View G;
    G.U = (const int *)(b + PL.U);
    G.V = (const int *)(b + PL.V);
    G.w = (const double *)(b + PL.w);
    G.row_off = (const int *)(b + PL.row_off);
    G.row_eid = (const int *)(b + PL.row_eid);
    G.ioff = (const int *)(b + PL.ioff);
    G.pairs = (const int2 *)(b + PL.pairs);
    G.nw = P.has_nw ? (const double *)(b + PL.nw) : nullptr;
    G.dinit = P.has_dinit ? (const double *)(b + PL.dinit) : nullptr;
    return G;
}

// Two schedules.  CTA mode: the CTA takes a chunk, stages its parent in
// shared memory and its groups share the chunk's subgraphs.  Group mode
// (whole-graph fits, one item per chunk): every group takes chunks on its
// own and reads the parent through L2, so no group idles behind another.
// Group-mode CTAs hold at most 256 threads (several per SM), which leaves
// the register budget of the larger networks unsplit.
template <bool GROUP, int MINB>
__global__ void __launch_bounds__(GROUP ? 256 : 512, MINB) k_batch(BatchLaunch L)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_chunk, s_next;
    Group g{(int)threadIdx.x / L.gsize, (int)threadIdx.x % L.gsize, L.gsize};
    const long long stage_bytes = L.stage ? pl_align(L.parent_bytes) : 0;
    unsigned char *gb = smem + stage_bytes + (long long)g.gid * group_bytes(L);
    double *d0 = (double *)gb;
    double *d1 = d0 + L.maxE;
    double *vd = d1 + L.maxE;
    double *red = vd + L.maxN;
    unsigned long long *slot = (unsigned long long *)(red + 2 * (L.gsize / 32));
    int *ks = (int *)(slot + 2);
    unsigned *eb = (unsigned *)(ks + (L.maxk > 0 ? L.maxk : 1));
    if (GROUP) {
        for (;;) {
            if (g.t == 0) slot[0] = (unsigned long long)atomicAdd(L.chunk_counter, 1);
            g.sync();
            const int c = (int)slot[0];
            g.sync();
            if (c >= L.nchunks) break;
            const Chunk ch = L.chunks[c];
            const ParentDesc P = L.parents[ch.parent];
            const ParentLayout PL = parent_layout(P.N, P.E, P.S, P.T, P.has_nw, P.has_dinit);
            const View G = view_of(P.data, PL, P);
            for (int i = 0; i < ch.count; ++i) fit_item(P, G, ch.first + i, g, d0, d1, vd, red, ks, slot, eb);
        }
        return;
    }
    int staged = -1;
    for (;;) {
        if (threadIdx.x == 0) s_chunk = atomicAdd(L.chunk_counter, 1);
        __syncthreads();
        const int c = s_chunk;
        if (c >= L.nchunks) break;
        const Chunk ch = L.chunks[c];
        const ParentDesc P = L.parents[ch.parent];
        const ParentLayout PL = parent_layout(P.N, P.E, P.S, P.T, P.has_nw, P.has_dinit);
        if (L.stage && ch.parent != staged) {
            const int4 *src = (const int4 *)P.data;
            int4 *dst = (int4 *)smem;
            for (long long q = threadIdx.x; q < PL.bytes / 16; q += blockDim.x) dst[q] = src[q];
            staged = ch.parent;
        }
        if (threadIdx.x == 0) s_next = 0;
        __syncthreads();
        const View G = view_of(L.stage ? smem : P.data, PL, P);
        for (;;) {
            if (g.t == 0) slot[0] = (unsigned long long)atomicAdd(&s_next, 1);
            g.sync();
            const int item = (int)slot[0];
            g.sync();
            if (item >= ch.count) break;
            fit_item(P, G, ch.first + item, g, d0, d1, vd, red, ks, slot, eb);
        }
        __syncthreads();
    }
}

template <bool GROUP, int MINB>
Status launch_mg(const BatchLaunch &L, int sms, cudaStream_t st)
{
    if (GROUP && L.gsize * L.groups > 256)
        return Status::Err(DRESSX_EINVAL, "group-mode batch CTAs hold at most 256 threads");
    size_t smem = batch_smem_bytes(L);
    DRESS_CUDA_TRY(cudaFuncSetAttribute(k_batch<GROUP, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    DRESS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch<GROUP, MINB>, L.gsize * L.groups, smem));
    if (per_sm < 1) return Status::Err(DRESSX_EUNSUPPORTED, "batch kernel does not fit on an SM");
    long long grid = (long long)per_sm * sms;
    // no more CTAs than there are chunks (group mode: chunks per CTA = groups)
    long long need = GROUP ? (L.nchunks + L.groups - 1) / L.groups : L.nchunks;
    if (grid > need) grid = need;
    count_launch(), k_batch<GROUP, MINB><<<(int)grid, L.gsize * L.groups, smem, st>>>(L);
    DRESS_CUDA_TRY(cudaGetLastError());
    return Status::Ok();
}

Status launch_any(const BatchLaunch &L, int sms, cudaStream_t st)
{
    if (L.per_group) return launch_mg<true, 1>(L, sms, st);
    if (L.min_ctas == 2) return launch_mg<false, 2>(L, sms, st);
    return launch_mg<false, 1>(L, sms, st);
}

// One whole-graph fit (ParentDesc of kind ITEM_PLAIN) by one cluster of
// CL_THREADS-thread CTAs.  Shared memory of a CTA: its slices of d, d_next
// and the vertex norms (per_e, per_e and per_n doubles), the warp slots, its
// two partials, and the tables of every CTA's slices.
constexpr int CL_THREADS = 512, CL_LB = 9;
constexpr int CL_MAX_CTAS = 16;

__global__ void __launch_bounds__(CL_THREADS, 1) k_fit_cluster(const ParentDesc *pp, int per_e, int per_n, int lnc)
{
    extern __shared__ __align__(16) unsigned char smem[];
    cg::cluster_group cl = cg::this_cluster();
    const int nc = (int)cl.num_blocks();
    double *s_d0 = (double *)smem;
    double *s_d1 = s_d0 + per_e;
    double *s_vd = s_d1 + per_e;
    double *wsl = s_vd + per_n;
    double *part = wsl + 2 * (CL_THREADS / 32);
    double **tab = (double **)(part + 2);          // [4][CL_MAX_CTAS]: d0, d1, vd, partials
    if ((int)threadIdx.x < nc) {
        const unsigned r = threadIdx.x;
        tab[0 * CL_MAX_CTAS + r] = cl.map_shared_rank(s_d0, r);
        tab[1 * CL_MAX_CTAS + r] = cl.map_shared_rank(s_d1, r);
        tab[2 * CL_MAX_CTAS + r] = cl.map_shared_rank(s_vd, r);
        tab[3 * CL_MAX_CTAS + r] = cl.map_shared_rank(part, r);
    }
    cl.sync();                                      // tables ready, every CTA running
    const ParentDesc P = *pp;
    const ParentLayout PL = parent_layout(P.N, P.E, P.S, P.T, P.has_nw, P.has_dinit);
    const View G = view_of(P.data, PL, P);
    const ClusterGroup g{(int)cl.block_rank() * CL_THREADS + (int)threadIdx.x, nc * CL_THREADS, wsl,
                         (double *const *)(tab + 3 * CL_MAX_CTAS), nc};
    const DArr d0{tab + 0 * CL_MAX_CTAS, CL_LB, lnc}, d1{tab + 1 * CL_MAX_CTAS, CL_LB, lnc},
        vd{tab + 2 * CL_MAX_CTAS, CL_LB, lnc};
    fit_item(P, G, 0, g, d0, d1, vd, nullptr, nullptr, nullptr, nullptr);
    cl.sync();                                      // no CTA leaves while others read its memory
}

Status launch_cluster_m(const ParentDesc *d_parent, int E, int N, int lnc, int sms, cudaStream_t st)
{
    const int nc = 1 << lnc, span = nc * CL_THREADS;
    const int per_e = ((E + span - 1) / span) * CL_THREADS, per_n = ((N + span - 1) / span) * CL_THREADS;
    const size_t smem = (size_t)(2 * per_e + per_n + 2 * (CL_THREADS / 32) + 2) * sizeof(double) +
                        4 * CL_MAX_CTAS * sizeof(double *);
    // attributes and the placement check are set up once per device and
    // cluster shape: the queries cost more than a small fit's whole launch
    int dev = 0;
    DRESS_CUDA_TRY(cudaGetDevice(&dev));
    static std::mutex mu;
    static std::map<std::tuple<int, int, size_t>, int> placeable;      // (device, CTAs, smem) -> clusters
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = placeable.find(std::make_tuple(dev, nc, smem));
        if (it != placeable.end()) {
            if (it->second < 1) return Status::Err(DRESSX_EUNSUPPORTED, "cluster fit does not fit the device");
        }
    }
    static std::mutex amu;
    static std::map<int, size_t> attr_smem;                             // device -> dynamic smem set
    {
        std::lock_guard<std::mutex> lk(amu);
        size_t &have = attr_smem[dev];
        if (have < smem) {
            DRESS_CUDA_TRY(cudaFuncSetAttribute(k_fit_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            DRESS_CUDA_TRY(cudaFuncSetAttribute(k_fit_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
            have = smem;
        }
    }
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)nc);
    cfg.blockDim = dim3(CL_THREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)nc;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int clusters = -1;
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = placeable.find(std::make_tuple(dev, nc, smem));
        if (it != placeable.end()) clusters = it->second;
    }
    if (clusters < 0) {
        if (cudaOccupancyMaxActiveClusters(&clusters, k_fit_cluster, &cfg) != cudaSuccess) {
            cudaGetLastError();
            clusters = 0;
        }
        std::lock_guard<std::mutex> lk(mu);
        placeable[std::make_tuple(dev, nc, smem)] = clusters;
    }
    if (clusters < 1) return Status::Err(DRESSX_EUNSUPPORTED, "cluster fit does not fit the device");
    count_launch();
    DRESS_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_fit_cluster, d_parent, per_e, per_n, lnc));
    (void)sms;
    return Status::Ok();
}

}  // namespace

size_t cluster_fit_smem_bytes(int E, int N, int lnc)
{
    const int span = (1 << lnc) * CL_THREADS;
    const int per_e = ((E + span - 1) / span) * CL_THREADS, per_n = ((N + span - 1) / span) * CL_THREADS;
    return (size_t)(2 * per_e + per_n + 2 * (CL_THREADS / 32) + 2) * sizeof(double) + 4 * CL_MAX_CTAS * sizeof(double *);
}

Status launch_cluster_fit(const ParentDesc *d_parent, int E, int N, int lnc, int sms, cudaStream_t st)
{
    if (lnc < 0 || (1 << lnc) > CL_MAX_CTAS) return Status::Err(DRESSX_EINVAL, "cluster size out of range");
    return launch_cluster_m(d_parent, E, N, lnc, sms, st);
}

long long batch_group_bytes(int maxE, int maxN, int maxk, int gsize)
{
    BatchLaunch L{};
    L.maxE = maxE;
    L.maxN = maxN;
    L.maxk = maxk;
    L.gsize = gsize;
    return group_bytes(L);
}

size_t batch_smem_bytes(const BatchLaunch &L)
{
    return (size_t)((L.stage ? pl_align(L.parent_bytes) : 0) + group_bytes(L) * L.groups);
}

Status launch_batch(const BatchLaunch &L, int sms, cudaStream_t st)
{
    if (L.nchunks <= 0) return Status::Ok();
    return launch_any(L, sms, st);
}

}  // namespace dress
