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
#include "batch.h"
#include "common.cuh"

namespace dress {
namespace {

__device__ __forceinline__ void cmx(double &a, double &b)
{
    double lo = fmin(a, b), hi = fmax(a, b);
    a = lo;
    b = hi;
}

// Bitonic network (single-direction form) on the first m registers.
template <int m, int M>
__device__ __forceinline__ void net(double (&a)[M])
{
#pragma unroll
    for (int k = 2; k <= m; k <<= 1) {
#pragma unroll
        for (int i = 0; i < m; ++i) {
            int j = i ^ (k - 1);
            if (j > i) cmx(a[i], a[j]);
        }
#pragma unroll
        for (int s = k >> 2; s > 0; s >>= 1) {
#pragma unroll
            for (int i = 0; i < m; ++i) {
                int j = i ^ s;
                if (j > i) cmx(a[i], a[j]);
            }
        }
    }
}

// Sorted KBN of the self term and the live ones among cnt stored terms
// (term(j, t) yields stored term j and whether it is alive) in a register
// network of Mi > cnt slots; dead and unused slots hold +inf.
template <int Mi, class Term>
__device__ __forceinline__ double net_sum(double self, int cnt, Term term)
{
    double a[Mi];
    a[0] = self;
    int n = 1;
#pragma unroll
    for (int j = 1; j < Mi; ++j) {
        a[j] = DRESS_INF;
        if (j <= cnt) {
            double t;
            if (term(j - 1, t)) {
                a[j] = t;
                ++n;
            }
        }
    }
    net<Mi, Mi>(a);
    double s = a[0], c = 0.0;
#pragma unroll
    for (int i = 1; i < Mi; ++i)
        if (i < n) kbn_step(s, c, a[i]);
    return dadd(s, c);
}

// The smallest network that holds the item: most items of sparse subgraphs
// have a handful of terms, and the cost of a network grows with its size.
template <int M, class Term>
__device__ __forceinline__ double item_sum(double self, int cnt, Term term)
{
    if (cnt == 0) return dadd(self, 0.0);
    if (cnt < 2) return net_sum<2>(self, cnt, term);
    if (M >= 4 && cnt < 4) return net_sum<(M >= 4 ? 4 : 2)>(self, cnt, term);
    if (M >= 8 && cnt < 8) return net_sum<(M >= 8 ? 8 : 2)>(self, cnt, term);
    if (M >= 16 && cnt < 16) return net_sum<(M >= 16 ? 16 : 2)>(self, cnt, term);
    return net_sum<M>(self, cnt, term);
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

template <int M>
__device__ void fit_item(const ParentDesc &P, const View &G, long long item,
                         const Group &g, double *d0, double *d1, double *vd, double *red, int *ks,
                         unsigned long long *slot)
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
    int live = 0;
    for (int e = g.t; e < E; e += g.size) {
        live += mk.alive(G.U[e]) && mk.alive(G.V[e]);
        d0[e] = P.has_dinit ? G.dinit[e] : 1.0;
    }
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
            vd[u] = dsqrt(item_sum<M>(dmul(4.0, mk.weight(u, G.nw)), deg, [&](int j, double &t) {
                const int e = G.row_eid[rb + j];
                if (!mk.alive(G.U[e] + G.V[e] - u)) return false;
                t = dmul(G.w[e], d0[e]);
                return true;
            }));
        }
        g.sync();
        double lmax = 0.0;
        for (int e = g.t; e < E; e += g.size) {
            const int u = G.U[e], v = G.V[e];
            if (!(mk.alive(u) && mk.alive(v))) continue;
            const double own = dmul(G.w[e], d0[e]);
            const double a4u = dmul(4.0, mk.weight(u, G.nw));
            const double self = P.fwd ? dadd(a4u, own) : dadd(dadd(a4u, dmul(4.0, mk.weight(v, G.nw))), dmul(2.0, own));
            const int pb = G.ioff[e], np = G.ioff[e + 1] - pb;
            const double num = item_sum<M>(self, np, [&](int j, double &t) {
                const int2 pr = G.pairs[pb + j];
                if (!mk.alive(G.U[pr.x] + G.V[pr.x] - u)) return false;
                t = dadd(dmul(G.w[pr.x], d0[pr.x]), dmul(G.w[pr.y], d0[pr.y]));
                return true;
            });
            const double den = dmul(vd[u], vd[v]);
            const double r = den > 0.0 ? ddiv(num, den) : 0.0;
            d1[e] = r;
            const double dd = fabs(dsub(d0[e], r));
            if (dd > lmax) lmax = dd;
        }
        const double m = group_max(g, lmax, red, (it & 1));
        last = m;
        double *t = d0;
        d0 = d1;
        d1 = t;
        g.sync();
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
    long long b = 8LL * (2LL * L.maxE + L.maxN) + 8LL * 2 * (L.gsize / 32) + 4LL * (L.maxk > 0 ? L.maxk : 1) + 16;
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
template <int M, bool GROUP, int MINB>
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
            for (int i = 0; i < ch.count; ++i) fit_item<M>(P, G, ch.first + i, g, d0, d1, vd, red, ks, slot);
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
            fit_item<M>(P, G, ch.first + item, g, d0, d1, vd, red, ks, slot);
        }
        __syncthreads();
    }
}

template <int M, bool GROUP, int MINB>
Status launch_mg(const BatchLaunch &L, int sms, cudaStream_t st)
{
    if (GROUP && L.gsize * L.groups > 256)
        return Status::Err(DRESSX_EINVAL, "group-mode batch CTAs hold at most 256 threads");
    size_t smem = batch_smem_bytes(L);
    DRESS_CUDA_TRY(cudaFuncSetAttribute(k_batch<M, GROUP, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    DRESS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch<M, GROUP, MINB>, L.gsize * L.groups, smem));
    if (per_sm < 1) return Status::Err(DRESSX_EUNSUPPORTED, "batch kernel does not fit on an SM");
    long long grid = (long long)per_sm * sms;
    // no more CTAs than there are chunks (group mode: chunks per CTA = groups)
    long long need = GROUP ? (L.nchunks + L.groups - 1) / L.groups : L.nchunks;
    if (grid > need) grid = need;
    count_launch(), k_batch<M, GROUP, MINB><<<(int)grid, L.gsize * L.groups, smem, st>>>(L);
    DRESS_CUDA_TRY(cudaGetLastError());
    return Status::Ok();
}

// Two CTAs per SM (64 registers a thread) only where the networks allow it.
template <int M>
Status launch_m(const BatchLaunch &L, int sms, cudaStream_t st)
{
    if (L.per_group) return launch_mg<M, true, 1>(L, sms, st);
    if (M <= 16 && L.min_ctas == 2) return launch_mg<M, false, (M <= 16 ? 2 : 1)>(L, sms, st);
    return launch_mg<M, false, 1>(L, sms, st);
}

}  // namespace

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
    switch (L.M) {
    case 2: return launch_m<2>(L, sms, st);
    case 4: return launch_m<4>(L, sms, st);
    case 8: return launch_m<8>(L, sms, st);
    case 16: return launch_m<16>(L, sms, st);
    case 32: return launch_m<32>(L, sms, st);
    default: return Status::Err(DRESSX_EUNSUPPORTED, "batch network size out of range");
    }
}

}  // namespace dress
