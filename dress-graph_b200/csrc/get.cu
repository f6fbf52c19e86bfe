// get.cu -- batched virtual-edge queries on a fitted graph.
//
// Reference: dress_get (libdress/src/dress.c:651-739) answers one (u, v)
// pair: the stored value of an existing edge, or, for a non-edge, the fixed
// point of the pair's own value with every other value frozen -- the sorted
// KBN sum of its common-neighbour terms w_ux d_ux + w_vx d_vx plus the
// self-loop constant, then a scalar iteration.  Here many pairs run at once:
//   k_get_scan    one thread per pair: the edge lookup (binary search of u's
//                 row), else the number of common neighbours (merge walk);
//   k_get_small   pairs with at most 31 common neighbours: the terms, sorted
//                 in a register network, and the iteration, one thread each;
//   k_get_fill / segmented_sort / k_get_large   longer pairs: the terms go to
//                 a slot per pair, are sorted per slot by the exact-histogram
//                 radix sort, and summed and iterated one thread each.
// Every operation is the reference's, in the same order, separately rounded.
#include <algorithm>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "engine.h"
#include "hist.h"

namespace dress {
namespace {

constexpr int SMALL = 32;                 // terms (common neighbours + self loop) in registers

struct GetGraph {
    int N, fwd, undirected;
    const int *off, *tgt, *eidx;
    const double *w, *d, *vd, *nw;       // nw null: unit vertex weights
};

__device__ __forceinline__ double ordered_to_double(unsigned long long k)
{
    unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffULL) : ~k;
    return __longlong_as_double((long long)b);
}

__device__ __forceinline__ double self_loop(const GetGraph &G, int u, int v)
{
    const double nu = G.nw ? G.nw[u] : 1.0, nv = G.nw ? G.nw[v] : 1.0;
    return G.fwd ? dmul(4.0, nu) : dadd(dmul(4.0, nu), dmul(4.0, nv));
}

// the pair's own fixed point from its intercept A (dress.c:713-738)
__device__ double iterate_pair(const GetGraph &G, int u, int v, double A, double ew, int max_iter, double eps)
{
    const double cf = G.fwd ? 1.0 : 2.0;
    const double cw = G.undirected ? dmul(2.0, ew) : ew;
    const double du2 = dmul(G.vd[u], G.vd[u]);
    const double dv2 = dmul(G.vd[v], G.vd[v]);
    if (du2 <= 0.0 || dv2 <= 0.0) return 0.0;
    double d = 1.0;
    for (int it = 0; it < max_iter; ++it) {
        const double wd = dmul(cw, d);
        const double den = dmul(dsqrt(dadd(du2, wd)), dsqrt(dadd(dv2, wd)));
        if (den <= 0.0) return 0.0;
        const double nx = ddiv(dadd(A, dmul(cf, wd)), den);
        if (fabs(dsub(nx, d)) <= eps) {
            d = nx;
            break;
        }
        d = nx;
    }
    return d;
}

__device__ __forceinline__ double term_of(const GetGraph &G, int eu, int ev)
{
    return dadd(dmul(G.w[eu], G.d[eu]), dmul(G.w[ev], G.d[ev]));
}

// cnt[i]: -1 for an existing edge (answered here), else common neighbours + 1
__global__ void k_get_scan(GetGraph G, long long n, const int *qu, const int *qv, int *cnt, double *out, int *bad)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int u = qu[i], v = qv[i];
        if (u < 0 || u >= G.N || v < 0 || v >= G.N) {
            atomicExch(bad, 1);
            cnt[i] = -1;
            out[i] = 0.0;
            continue;
        }
        int lo = G.off[u], hi = G.off[u + 1] - 1;
        int found = -1;
        while (lo <= hi) {
            const int mid = lo + (hi - lo) / 2;
            const int nb = G.tgt[mid];
            if (nb == v) { found = mid; break; }
            if (nb < v) lo = mid + 1;
            else hi = mid - 1;
        }
        if (found >= 0) {
            out[i] = G.d[G.eidx[found]];
            cnt[i] = -1;
            continue;
        }
        int c = 0;
        int iu = G.off[u], iu_end = G.off[u + 1];
        int iv = G.off[v], iv_end = G.off[v + 1];
        while (iu < iu_end && iv < iv_end) {
            const int x = G.tgt[iu], y = G.tgt[iv];
            c += x == y;
            iu += (x <= y);
            iv += (x >= y);
        }
        cnt[i] = c + 1;
    }
}

__global__ void k_get_small(GetGraph G, long long n, const int *qu, const int *qv, const int *cnt, const double *ew,
                            double ew0, int max_iter, double eps, double *out)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int c = cnt[i];
        if (c < 0 || c > SMALL) continue;
        const int u = qu[i], v = qv[i];
        double a[SMALL];
#pragma unroll
        for (int k = 0; k < SMALL; ++k) a[k] = DRESS_INF;
        int m = 0;
        int iu = G.off[u], iu_end = G.off[u + 1];
        int iv = G.off[v], iv_end = G.off[v + 1];
        while (iu < iu_end && iv < iv_end) {
            const int x = G.tgt[iu], y = G.tgt[iv];
            if (x == y) {
                const double t = term_of(G, G.eidx[iu], G.eidx[iv]);
#pragma unroll
                for (int k = 0; k < SMALL; ++k)
                    if (k == m) a[k] = t;
                ++m;
            }
            iu += (x <= y);
            iv += (x >= y);
        }
        const double sl = self_loop(G, u, v);
#pragma unroll
        for (int k = 0; k < SMALL; ++k)
            if (k == m) a[k] = sl;
        sort_regs<SMALL>(a);
        const double A = kbn_regs<SMALL>(a, c);
        out[i] = iterate_pair(G, u, v, A, ew ? ew[i] : ew0, max_iter, eps);
    }
}

// the terms of the long pairs into their slots (order-preserving image)
__global__ void k_get_fill(GetGraph G, long long n, const int *qu, const int *qv, const int *cnt,
                           const long long *slot, unsigned long long *keys)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int c = cnt[i];
        if (c <= SMALL) continue;
        const int u = qu[i], v = qv[i];
        unsigned long long *k = keys + slot[i];
        int m = 0;
        int iu = G.off[u], iu_end = G.off[u + 1];
        int iv = G.off[v], iv_end = G.off[v + 1];
        while (iu < iu_end && iv < iv_end) {
            const int x = G.tgt[iu], y = G.tgt[iv];
            if (x == y) k[m++] = (unsigned long long)__double_as_longlong(term_of(G, G.eidx[iu], G.eidx[iv]));
            iu += (x <= y);
            iv += (x >= y);
        }
        k[m] = (unsigned long long)__double_as_longlong(self_loop(G, u, v));
    }
}

__global__ void k_get_large(GetGraph G, long long n, const int *qu, const int *qv, const int *cnt,
                            const long long *slot, const unsigned long long *sorted, const double *ew, double ew0,
                            int max_iter, double eps, double *out)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int c = cnt[i];
        if (c <= SMALL) continue;
        const unsigned long long *k = sorted + slot[i];
        double s = ordered_to_double(k[0]), cc = 0.0;
        for (int t = 1; t < c; ++t) kbn_step(s, cc, ordered_to_double(k[t]));
        out[i] = iterate_pair(G, qu[i], qv[i], dadd(s, cc), ew ? ew[i] : ew0, max_iter, eps);
    }
}

template <class T>
Status upload(DevBuf<T> &b, const T *host, size_t n, cudaStream_t st)
{
    DRESS_TRY(b.alloc(n > 0 ? n : 1, st));
    if (n) DRESS_CUDA_TRY(counted_memcpy(b.get(), host, n * sizeof(T), cudaMemcpyHostToDevice, st));
    return Status::Ok();
}

}  // namespace

Status get_batch(p_dress_graph_t g, const int *u, const int *v, long long n, int max_iterations, double epsilon,
                 const double *edge_weights, double edge_weight, double *out, const Ctx &ctx)
{
    if (!g || n < 0 || (n > 0 && (!u || !v || !out))) return Status::Err(DRESSX_EINVAL, "bad arguments");
    if (n == 0) return Status::Ok();
    const int N = g->N, E = g->E;
    const long long S = N > 0 ? g->adj_offset[N] : 0;
    if (N <= 0) return Status::Err(DRESSX_EINVAL, "query on an empty graph");
    cudaStream_t st = ctx.st;
    const int sms = ctx.num_sms;
    DRESS_CUDA_TRY(cudaSetDevice(ctx.device));
    DevBuf<int> d_off, d_tgt, d_eidx, d_u, d_v, d_cnt, d_bad;
    DevBuf<double> d_w, d_d, d_vd, d_nw, d_ew, d_out;
    DRESS_TRY(upload(d_off, g->adj_offset, (size_t)N + 1, st));
    DRESS_TRY(upload(d_tgt, g->adj_target, (size_t)S, st));
    DRESS_TRY(upload(d_eidx, g->adj_edge_idx, (size_t)S, st));
    DRESS_TRY(upload(d_w, g->edge_weight, (size_t)E, st));
    DRESS_TRY(upload(d_d, g->edge_dress, (size_t)E, st));
    DRESS_TRY(upload(d_vd, g->vertex_dress, (size_t)N, st));
    if (g->NW) DRESS_TRY(upload(d_nw, g->NW, (size_t)N, st));
    DRESS_TRY(upload(d_u, u, (size_t)n, st));
    DRESS_TRY(upload(d_v, v, (size_t)n, st));
    if (edge_weights) DRESS_TRY(upload(d_ew, edge_weights, (size_t)n, st));
    DRESS_TRY(d_cnt.alloc((size_t)n, st));
    DRESS_TRY(d_out.alloc((size_t)n, st));
    DRESS_TRY(d_bad.alloc(1, st));
    DRESS_CUDA_TRY(cudaMemsetAsync(d_bad.get(), 0, sizeof(int), st));
    GetGraph G{N, g->variant == DRESS_VARIANT_FORWARD || g->variant == DRESS_VARIANT_BACKWARD,
               g->variant == DRESS_VARIANT_UNDIRECTED, d_off.get(), d_tgt.get(), d_eidx.get(),
               d_w.get(), d_d.get(), d_vd.get(), g->NW ? d_nw.get() : nullptr};
    const unsigned grid = (unsigned)std::min<long long>((n + 127) / 128, 16LL * sms);
    count_launch(), k_get_scan<<<grid, 128, 0, st>>>(G, n, d_u.get(), d_v.get(), d_cnt.get(), d_out.get(), d_bad.get());
    count_launch(), k_get_small<<<grid, 128, 0, st>>>(G, n, d_u.get(), d_v.get(), d_cnt.get(),
                                                      edge_weights ? d_ew.get() : nullptr, edge_weight,
                                                      max_iterations, epsilon, d_out.get());
    // pairs with more terms: slots, per-slot sort, sums
    std::vector<int> cnt((size_t)n);
    int bad = 0;
    DRESS_CUDA_TRY(counted_memcpy(cnt.data(), d_cnt.get(), (size_t)n * sizeof(int), cudaMemcpyDeviceToHost, st));
    DRESS_CUDA_TRY(counted_memcpy(&bad, d_bad.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
    DRESS_CUDA_TRY(cudaStreamSynchronize(st));
    if (bad) return Status::Err(DRESSX_EINVAL, "query vertex out of range");
    std::vector<long long> slot((size_t)n, 0), begin, len;
    long long total = 0;
    for (long long i = 0; i < n; ++i)
        if (cnt[(size_t)i] > SMALL) {
            slot[(size_t)i] = total;
            begin.push_back(total);
            len.push_back(cnt[(size_t)i]);
            total += cnt[(size_t)i];
        }
    if (total > 0) {
        DevBuf<long long> d_slot;
        DevBuf<unsigned long long> d_keys, d_alt;
        DRESS_TRY(upload(d_slot, slot.data(), (size_t)n, st));
        DRESS_TRY(d_keys.alloc((size_t)total, st));
        DRESS_TRY(d_alt.alloc((size_t)total, st));
        count_launch(), k_get_fill<<<grid, 128, 0, st>>>(G, n, d_u.get(), d_v.get(), d_cnt.get(), d_slot.get(),
                                                         d_keys.get());
        unsigned long long *sorted = nullptr;
        DRESS_TRY(segmented_sort(d_keys.get(), d_alt.get(), begin, len, &sorted, st, sms));
        count_launch(), k_get_large<<<grid, 128, 0, st>>>(G, n, d_u.get(), d_v.get(), d_cnt.get(), d_slot.get(), sorted,
                                                          edge_weights ? d_ew.get() : nullptr, edge_weight,
                                                          max_iterations, epsilon, d_out.get());
        DRESS_CUDA_TRY(cudaGetLastError());
        DRESS_CUDA_TRY(counted_memcpy(out, d_out.get(), (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, st));
        DRESS_CUDA_TRY(cudaStreamSynchronize(st));
        return Status::Ok();
    }
    DRESS_CUDA_TRY(cudaGetLastError());
    DRESS_CUDA_TRY(counted_memcpy(out, d_out.get(), (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, st));
    DRESS_CUDA_TRY(cudaStreamSynchronize(st));
    return Status::Ok();
}

}  // namespace dress

using namespace dress;

extern "C" int dressx_get_batch(p_dress_graph_t g, const int *u, const int *v, int64_t n, int max_iterations,
                                double epsilon, const double *edge_weights, double edge_weight, double *out)
{
    Engine &en = engine();
    std::lock_guard<std::mutex> lk(en.mu);
    Status s = en.init();
    if (s.ok()) s = get_batch(g, u, v, (long long)n, max_iterations, epsilon, edge_weights, edge_weight, out, en.ctx);
    set_last_error(s);
    return s.code;
}
