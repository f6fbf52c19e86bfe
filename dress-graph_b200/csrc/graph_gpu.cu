// graph_gpu.cu -- dress_init_graph built on the GPU (dressx_init_graph).
//
// Same contract and bit-identical output as the host build (graph_host.cpp)
// and the reference (libdress/src/dress.c:103-427): the variant CSR with rows
// ascending by neighbour id, ties in insertion order; variant weights; the
// optional common-neighbour tables; every edge value 1.0.  The host build
// orders rows with two stable counting passes; here one stable radix sort of
// (row, neighbour) keys does it on the device:
//   raw slots    u->v for every edge (and v->u when undirected), in insertion
//                order, sorted stably by (row, neighbour);
//   variants     UNDIRECTED / FORWARD keep the raw order; BACKWARD re-sorts the
//                reversed slots; DIRECTED looks each slot's reciprocal up by
//                the reference's bisection over the sorted raw row (same probe
//                sequence, so the same entry among repeated edges), emits the
//                slot and, without a reciprocal, its reverse right after it,
//                and re-sorts;
//   CSR          offsets, targets, edge ids and w-bar from the sorted slots;
//   intercepts   the merge walk of libdress/src/dress.c:307-363, per edge.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#include "dress_b200.h"
#include "engine.h"
#include "hist.h"

namespace dress {
namespace {

constexpr unsigned long long NO_SLOT = ~0ULL;   // sorts after every real slot

__device__ __forceinline__ unsigned long long slot_key(int row, int x)
{
    return ((unsigned long long)(unsigned)row << 32) | (unsigned)x;
}

__global__ void k_check(int N, int E, const int *U, const int *V, int *bad)
{
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += gridDim.x * blockDim.x)
        if (U[e] < 0 || U[e] >= N || V[e] < 0 || V[e] >= N) atomicExch(bad, 1);
}

// raw slots in insertion order: slot 2e = U->V, 2e+1 = V->U (undirected), else slot e
__global__ void k_raw_slots(int E, int und, const int *U, const int *V, unsigned long long *key, unsigned *id)
{
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += gridDim.x * blockDim.x) {
        if (und) {
            key[2LL * e] = slot_key(U[e], V[e]);
            id[2LL * e] = 2u * (unsigned)e;
            key[2LL * e + 1] = slot_key(V[e], U[e]);
            id[2LL * e + 1] = 2u * (unsigned)e + 1u;
        } else {
            key[e] = slot_key(U[e], V[e]);
            id[e] = (unsigned)e;
        }
    }
}

__global__ void k_row_count(long long R, const unsigned long long *key, int *deg)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < R; i += (long long)gridDim.x * blockDim.x)
        if (key[i] != NO_SLOT) atomicAdd(&deg[(int)(key[i] >> 32)], 1);
}

// BACKWARD: the reversed slot of every raw slot, in raw order
__global__ void k_backward(long long R, const unsigned long long *key, const unsigned *id, unsigned long long *vkey,
                           unsigned *vid)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < R; i += (long long)gridDim.x * blockDim.x) {
        const int row = (int)(key[i] >> 32), x = (int)(key[i] & 0xffffffffu);
        vkey[i] = slot_key(x, row);
        vid[i] = id[i];
    }
}

// DIRECTED: slot 2i (the edge itself, w-bar = w + w of the reciprocal when
// there is one) and slot 2i+1 (its reverse when there is none)
__global__ void k_directed(long long R, const unsigned long long *key, const unsigned *id, const long long *roff,
                           const double *W, unsigned long long *vkey, unsigned *vedge, double *vw)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < R; i += (long long)gridDim.x * blockDim.x) {
        const int u = (int)(key[i] >> 32), v = (int)(key[i] & 0xffffffffu);
        const unsigned e = id[i];
        const double w = W ? W[e] : 1.0;
        long long lo = roff[v], hi = roff[v + 1] - 1, r = -1;      // reciprocal v->u
        while (lo <= hi) {
            const long long mid = lo + (hi - lo) / 2;
            const int x = (int)(key[mid] & 0xffffffffu);
            if (x == u) { r = mid; break; }
            if (x < u) lo = mid + 1;
            else hi = mid - 1;
        }
        vkey[2 * i] = slot_key(u, v);
        vedge[2 * i] = e;
        vw[2 * i] = r >= 0 ? w + (W ? W[id[r]] : 1.0) : w;
        vkey[2 * i + 1] = r >= 0 ? NO_SLOT : slot_key(v, u);
        vedge[2 * i + 1] = e;
        vw[2 * i + 1] = w;
    }
}

__global__ void k_iota(long long n, unsigned *out)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = (unsigned)i;
}

// the CSR from the sorted slots; wmode 0: w-bar = 2w, 1: w, 2: per-slot weights
__global__ void k_csr(long long S, int und_ids, const unsigned long long *key, const unsigned *id,
                      const unsigned *vedge, const double *vw, const double *W, int wmode, int *tgt, int *eidx,
                      double *ew)
{
    for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < S; s += (long long)gridDim.x * blockDim.x) {
        const unsigned q = id[s];
        const int e = vedge ? (int)vedge[q] : (und_ids ? (int)(q >> 1) : (int)q);
        tgt[s] = (int)(key[s] & 0xffffffffu);
        eidx[s] = e;
        double w;
        if (wmode == 2) w = vw[q];
        else {
            const double w0 = W ? W[e] : 1.0;
            w = wmode == 0 ? 2.0 * w0 : w0;
        }
        ew[e] = w;                  // every slot of an edge carries the same w-bar
    }
}

// common-neighbour tables by the merge walk
template <bool FILL>
__global__ void k_intercepts(int E, const int *U, const int *V, const int *off, const int *tgt, const int *eidx,
                             int *cnt, const long long *ioff, int *ux, int *vx)
{
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += gridDim.x * blockDim.x) {
        int iu = off[U[e]], iu_end = off[U[e] + 1];
        int iv = off[V[e]], iv_end = off[V[e] + 1];
        long long o = FILL ? ioff[e] : 0;
        int c = 0;
        while (iu < iu_end && iv < iv_end) {
            const int x = tgt[iu], y = tgt[iv];
            if (x == y) {
                if (FILL) {
                    ux[o] = eidx[iu];
                    vx[o] = eidx[iv];
                    ++o;
                } else {
                    ++c;
                }
            }
            iu += (x <= y);
            iv += (x >= y);
        }
        if (!FILL) cnt[e] = c;
    }
}

inline unsigned grid1(long long n, int sms) { return (unsigned)std::max<long long>(1, std::min<long long>((n + 255) / 256, 32LL * sms)); }

template <class T>
T *xmalloc(size_t n) { return (T *)std::malloc((n ? n : 1) * sizeof(T)); }

void fill_ones(double *p, size_t n)
{
    const size_t chunk = 1 << 22;
    if (n <= chunk) {
        std::fill(p, p + n, 1.0);
        return;
    }
    std::vector<std::thread> th;
    const int nt = 8;
    for (int t = 0; t < nt; ++t)
        th.emplace_back([=] {
            const size_t a = n * t / nt, b = n * (t + 1) / nt;
            std::fill(p + a, p + b, 1.0);
        });
    for (auto &x : th) x.join();
}

Status build(p_dress_graph_t g, const Ctx &ctx)
{
    cudaStream_t st = ctx.st;
    const int sms = ctx.num_sms;
    const int N = g->N, E = g->E;
    const dress_variant_t variant = g->variant;
    const bool und = variant == DRESS_VARIANT_UNDIRECTED;
    DRESS_CUDA_TRY(cudaSetDevice(ctx.device));

    DevBuf<int> d_U, d_V, d_bad, d_deg;
    DevBuf<double> d_W;
    DRESS_TRY(d_U.alloc((size_t)std::max(E, 1), st));
    DRESS_TRY(d_V.alloc((size_t)std::max(E, 1), st));
    DRESS_TRY(d_bad.alloc(1, st));
    if (E) {
        DRESS_CUDA_TRY(counted_memcpy(d_U.get(), g->U, (size_t)E * 4, cudaMemcpyHostToDevice, st));
        DRESS_CUDA_TRY(counted_memcpy(d_V.get(), g->V, (size_t)E * 4, cudaMemcpyHostToDevice, st));
    }
    if (g->W) {
        DRESS_TRY(d_W.alloc((size_t)std::max(E, 1), st));
        if (E) DRESS_CUDA_TRY(counted_memcpy(d_W.get(), g->W, (size_t)E * 8, cudaMemcpyHostToDevice, st));
    }
    DRESS_CUDA_TRY(cudaMemsetAsync(d_bad.get(), 0, sizeof(int), st));
    if (E) count_launch(), k_check<<<grid1(E, sms), 256, 0, st>>>(N, E, d_U.get(), d_V.get(), d_bad.get());
    int bad = 0;
    DRESS_CUDA_TRY(counted_memcpy(&bad, d_bad.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
    DRESS_CUDA_TRY(cudaStreamSynchronize(st));
    if (bad) return Status::Err(DRESSX_EINVAL, "edge endpoint out of range");

    // raw slots, sorted stably by (row, neighbour)
    const long long R = und ? 2LL * E : E;
    DevBuf<unsigned long long> k0, k1;
    DevBuf<unsigned> i0, i1;
    DRESS_TRY(k0.alloc((size_t)std::max(R, 1LL), st));
    DRESS_TRY(k1.alloc((size_t)std::max(R, 1LL), st));
    DRESS_TRY(i0.alloc((size_t)std::max(R, 1LL), st));
    DRESS_TRY(i1.alloc((size_t)std::max(R, 1LL), st));
    if (E) count_launch(), k_raw_slots<<<grid1(E, sms), 256, 0, st>>>(E, und, d_U.get(), d_V.get(), k0.get(), i0.get());
    unsigned long long *rk = k0.get();
    unsigned *ri = i0.get();
    if (R) DRESS_TRY(sort_pairs(k0.get(), k1.get(), i0.get(), i1.get(), R, &rk, &ri, st, sms));

    // the variant slots (keys, payload)
    const unsigned long long *vk = rk;
    const unsigned *vi = ri;
    const unsigned *vedge = nullptr;
    const double *vw = nullptr;
    long long S = R;
    int wmode = und ? 0 : 1;
    DevBuf<unsigned long long> vk0, vk1;
    DevBuf<unsigned> vi0, vi1, d_vedge;
    DevBuf<double> d_vw;
    DevBuf<long long> d_roff, d_tmp;
    if (variant == DRESS_VARIANT_BACKWARD && R) {
        DRESS_TRY(vk0.alloc((size_t)R, st));
        DRESS_TRY(vk1.alloc((size_t)R, st));
        DRESS_TRY(vi0.alloc((size_t)R, st));
        DRESS_TRY(vi1.alloc((size_t)R, st));
        count_launch(), k_backward<<<grid1(R, sms), 256, 0, st>>>(R, rk, ri, vk0.get(), vi0.get());
        unsigned long long *sk;
        unsigned *si;
        DRESS_TRY(sort_pairs(vk0.get(), vk1.get(), vi0.get(), vi1.get(), R, &sk, &si, st, sms));
        vk = sk;
        vi = si;
    } else if (variant == DRESS_VARIANT_DIRECTED && R) {
        // raw row offsets for the reciprocal lookups
        DRESS_TRY(d_deg.alloc((size_t)N + 1, st));
        DRESS_TRY(d_roff.alloc((size_t)N + 1, st));
        DRESS_TRY(d_tmp.alloc(scan_tmp_elems(N), st));
        DRESS_CUDA_TRY(cudaMemsetAsync(d_deg.get(), 0, ((size_t)N + 1) * sizeof(int), st));
        count_launch(), k_row_count<<<grid1(R, sms), 256, 0, st>>>(R, rk, d_deg.get());
        DRESS_TRY(exclusive_scan_i32(d_deg.get(), d_roff.get(), N, d_tmp.get(), st));
        DRESS_TRY(vk0.alloc(2 * (size_t)R, st));
        DRESS_TRY(vk1.alloc(2 * (size_t)R, st));
        DRESS_TRY(vi0.alloc(2 * (size_t)R, st));
        DRESS_TRY(vi1.alloc(2 * (size_t)R, st));
        DRESS_TRY(d_vedge.alloc(2 * (size_t)R, st));
        DRESS_TRY(d_vw.alloc(2 * (size_t)R, st));
        count_launch(), k_directed<<<grid1(R, sms), 256, 0, st>>>(R, rk, ri, d_roff.get(), g->W ? d_W.get() : nullptr,
                                                                   vk0.get(), d_vedge.get(), d_vw.get());
        // payload = emission index, in emission order
        count_launch(), k_iota<<<grid1(2 * R, sms), 256, 0, st>>>(2 * R, vi0.get());
        unsigned long long *sk;
        unsigned *si;
        DRESS_TRY(sort_pairs(vk0.get(), vk1.get(), vi0.get(), vi1.get(), 2 * R, &sk, &si, st, sms));
        vk = sk;
        vi = si;
        vedge = d_vedge.get();
        vw = d_vw.get();
        wmode = 2;
        // the real slots sort ahead of the absent ones
        DevBuf<int> d_cnt;
        DRESS_TRY(d_cnt.alloc((size_t)N + 1, st));
        DRESS_CUDA_TRY(cudaMemsetAsync(d_cnt.get(), 0, ((size_t)N + 1) * sizeof(int), st));
        count_launch(), k_row_count<<<grid1(2 * R, sms), 256, 0, st>>>(2 * R, vk, d_cnt.get());
        std::vector<int> cnt((size_t)N);
        DRESS_CUDA_TRY(counted_memcpy(cnt.data(), d_cnt.get(), (size_t)N * 4, cudaMemcpyDeviceToHost, st));
        DRESS_CUDA_TRY(cudaStreamSynchronize(st));
        S = 0;
        for (int c : cnt) S += c;
    }

    // CSR
    DevBuf<int> d_vdeg, d_tgt, d_eidx, d_off32;
    DevBuf<long long> d_off, d_tmp2;
    DevBuf<double> d_ew;
    DRESS_TRY(d_vdeg.alloc((size_t)N + 1, st));
    DRESS_TRY(d_off.alloc((size_t)N + 1, st));
    DRESS_TRY(d_tmp2.alloc(scan_tmp_elems(N), st));
    DRESS_TRY(d_tgt.alloc((size_t)std::max(S, 1LL), st));
    DRESS_TRY(d_eidx.alloc((size_t)std::max(S, 1LL), st));
    DRESS_TRY(d_ew.alloc((size_t)std::max(E, 1), st));
    DRESS_CUDA_TRY(cudaMemsetAsync(d_vdeg.get(), 0, ((size_t)N + 1) * sizeof(int), st));
    if (S) {
        count_launch(), k_row_count<<<grid1(S, sms), 256, 0, st>>>(S, vk, d_vdeg.get());
        count_launch(), k_csr<<<grid1(S, sms), 256, 0, st>>>(S, und, vk, vi, vedge, vw, g->W ? d_W.get() : nullptr,
                                                             wmode, d_tgt.get(), d_eidx.get(), d_ew.get());
    }
    DRESS_TRY(exclusive_scan_i32(d_vdeg.get(), d_off.get(), N, d_tmp2.get(), st));
    std::vector<long long> off64((size_t)N + 1);
    DRESS_CUDA_TRY(counted_memcpy(off64.data(), d_off.get(), ((size_t)N + 1) * 8, cudaMemcpyDeviceToHost, st));

    g->adj_offset = xmalloc<int>((size_t)N + 1);
    g->adj_target = xmalloc<int>((size_t)S);
    g->adj_edge_idx = xmalloc<int>((size_t)S);
    g->edge_weight = xmalloc<double>((size_t)E);
    if (S) {
        DRESS_CUDA_TRY(counted_memcpy(g->adj_target, d_tgt.get(), (size_t)S * 4, cudaMemcpyDeviceToHost, st));
        DRESS_CUDA_TRY(counted_memcpy(g->adj_edge_idx, d_eidx.get(), (size_t)S * 4, cudaMemcpyDeviceToHost, st));
    }
    if (E) DRESS_CUDA_TRY(counted_memcpy(g->edge_weight, d_ew.get(), (size_t)E * 8, cudaMemcpyDeviceToHost, st));
    DRESS_CUDA_TRY(cudaStreamSynchronize(st));
    int maxdeg = 0;
    for (int i = 0; i <= N; ++i) g->adj_offset[i] = (int)off64[(size_t)i];
    for (int i = 0; i < N; ++i) maxdeg = std::max(maxdeg, g->adj_offset[i + 1] - g->adj_offset[i]);
    g->max_degree = maxdeg;

    if (g->precompute_intercepts) {
        DevBuf<int> d_offi, d_cnt, d_ux, d_vx;
        DevBuf<long long> d_io, d_tmp3;
        DRESS_TRY(d_offi.alloc((size_t)N + 1, st));
        DRESS_CUDA_TRY(counted_memcpy(d_offi.get(), g->adj_offset, ((size_t)N + 1) * 4, cudaMemcpyHostToDevice, st));
        DRESS_TRY(d_cnt.alloc((size_t)std::max(E, 1), st));
        DRESS_TRY(d_io.alloc((size_t)E + 1, st));
        DRESS_TRY(d_tmp3.alloc(scan_tmp_elems(E), st));
        if (E) count_launch(), k_intercepts<false><<<grid1(E, sms), 256, 0, st>>>(E, d_U.get(), d_V.get(), d_offi.get(),
                                                                                 d_tgt.get(), d_eidx.get(), d_cnt.get(),
                                                                                 nullptr, nullptr, nullptr);
        DRESS_TRY(exclusive_scan_i32(d_cnt.get(), d_io.get(), E, d_tmp3.get(), st));
        std::vector<long long> io((size_t)E + 1);
        DRESS_CUDA_TRY(counted_memcpy(io.data(), d_io.get(), ((size_t)E + 1) * 8, cudaMemcpyDeviceToHost, st));
        DRESS_CUDA_TRY(cudaStreamSynchronize(st));
        const long long T = io[(size_t)E];
        if (T > 0x7fffffffLL) return Status::Err(DRESSX_EUNSUPPORTED, "intercept tables beyond int range");
        DRESS_TRY(d_ux.alloc((size_t)std::max(T, 1LL), st));
        DRESS_TRY(d_vx.alloc((size_t)std::max(T, 1LL), st));
        if (E) count_launch(), k_intercepts<true><<<grid1(E, sms), 256, 0, st>>>(E, d_U.get(), d_V.get(), d_offi.get(),
                                                                                d_tgt.get(), d_eidx.get(), nullptr,
                                                                                d_io.get(), d_ux.get(), d_vx.get());
        g->intercept_offset = xmalloc<int>((size_t)E + 1);
        for (int e = 0; e <= E; ++e) g->intercept_offset[e] = (int)io[(size_t)e];
        g->intercept_edge_ux = xmalloc<int>((size_t)T);
        g->intercept_edge_vx = xmalloc<int>((size_t)T);
        if (T) {
            DRESS_CUDA_TRY(counted_memcpy(g->intercept_edge_ux, d_ux.get(), (size_t)T * 4, cudaMemcpyDeviceToHost, st));
            DRESS_CUDA_TRY(counted_memcpy(g->intercept_edge_vx, d_vx.get(), (size_t)T * 4, cudaMemcpyDeviceToHost, st));
        }
        DRESS_CUDA_TRY(cudaStreamSynchronize(st));
    }
    return Status::Ok();
}

}  // namespace
}  // namespace dress

using namespace dress;

extern "C" p_dress_graph_t dressx_init_graph(int N, int E, int *U, int *V, double *W, double *NW,
                                            dress_variant_t variant, int precompute_intercepts)
{
    if (N < 0 || E < 0 || (E > 0 && (!U || !V))) return nullptr;
    p_dress_graph_t g = (p_dress_graph_t)std::calloc(1, sizeof(dress_graph_t));
    if (!g) return nullptr;
    g->variant = variant;
    g->N = N;
    g->E = E;
    g->U = U;
    g->V = V;
    g->W = W;
    g->precompute_intercepts = precompute_intercepts;
    Status s;
    {
        Engine &en = engine();
        std::lock_guard<std::mutex> lk(en.mu);
        s = en.init();
        if (s.ok()) s = build(g, en.ctx);
    }
    if (!s.ok()) {
        set_last_error(s);
        std::free(g->adj_offset);
        std::free(g->adj_target);
        std::free(g->adj_edge_idx);
        std::free(g->edge_weight);
        std::free(g->intercept_offset);
        std::free(g->intercept_edge_ux);
        std::free(g->intercept_edge_vx);
        std::free(g);
        return nullptr;                       // the caller keeps U, V, W, NW
    }
    g->vertex_dress = xmalloc<double>((size_t)N);
    if (NW) {
        g->NW = NW;
    } else {
        g->NW = xmalloc<double>((size_t)N);
        fill_ones(g->NW, (size_t)N);
    }
    g->edge_dress = xmalloc<double>((size_t)E);
    g->edge_dress_next = xmalloc<double>((size_t)E);
    fill_ones(g->edge_dress, (size_t)E);
    fill_ones(g->edge_dress_next, (size_t)E);
    set_last_error(Status::Ok());
    return g;
}
