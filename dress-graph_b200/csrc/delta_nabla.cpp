// delta_nabla.cpp -- Delta^k / Nabla^k requests and the legacy entry points.
//
// Reference drivers: libdress/src/delta_dress_impl.c:171-318 and
// libdress/src/nabla_dress_impl.c:142-311; public wrappers
// libdress/src/cuda/delta_dress_cuda.c:24-85, nabla_dress_cuda.c:24-85.
// The argument meaning is unchanged: subsets (ordered tuples) are ranked
// lexicographically, rank s is processed when s % stride == offset, with
// n_samples > 0 a sorted, de-duplicated LCG sample of the stride's ranks is
// processed, k == 0 fits the caller's graph in place, k >= N gives an empty
// histogram, edgeless subgraphs are skipped, and the histogram is the exact
// (value, count) list ascending by value.
//
// Requests whose parent fits the batched kernel (rows of at most 31
// neighbours, per-subgraph state within shared memory) are packed into one
// persistent launch; any other request runs through the per-subgraph path:
// host-built subgraph + single-graph GPU fit (the reference's structure,
// which is also the "plain per-fit launch loop" the batched engine is
// measured against).  Histograms are always built on the GPU.
#include <algorithm>
#include <cmath>
#include <map>
#include <memory>
#include <mutex>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#include "batch.h"
#include "engine.h"
#include "hist.h"
#include "host_par.h"

namespace dress {

long long binom_h(int n, int k)
{
    if (k < 0 || k > n) return 0;
    if (k == 0 || k == n) return 1;
    if (k > n - k) k = n - k;
    long long r = 1;
    for (int i = 0; i < k; ++i) r = r * (n - i) / (i + 1);
    return r;
}

long long perm_h(int n, int k)
{
    if (k < 0 || k > n) return 0;
    long long r = 1;
    for (int i = 0; i < k; ++i) r *= (n - i);
    return r;
}

void merge_walk_pairs(p_dress_graph_t g, std::vector<int> &ioff, std::vector<int> &pairs, int &maxdeg, bool &dup)
{
    const int N = g->N, E = g->E;
    const int *off = g->adj_offset, *tg = g->adj_target, *ei = g->adj_edge_idx;
    maxdeg = 0;
    dup = false;
    for (int u = 0; u < N; ++u) {
        maxdeg = std::max(maxdeg, off[u + 1] - off[u]);
        for (int s = off[u] + 1; s < off[u + 1]; ++s) dup |= tg[s] == tg[s - 1];
    }
    ioff.assign((size_t)E + 1, 0);
    pairs.clear();
    if (!dup) {
        // Rows without repeated neighbours: the intersection of rows U[e]
        // and V[e] is found by marking U[e]'s row and scanning V[e]'s in
        // order -- the merge walk's pairs, in its order (ascending common
        // neighbour), without its branches.  Edges are taken grouped by
        // U[e], so a row is marked once.
        std::vector<int> first((size_t)N + 1, 0), byu((size_t)E), slot_of((size_t)N), stamp((size_t)N, -1);
        for (int e = 0; e < E; ++e) ++first[(size_t)g->U[e] + 1];
        for (int u = 0; u < N; ++u) first[(size_t)u + 1] += first[(size_t)u];
        {
            std::vector<int> cur(first.begin(), first.end() - 1);
            for (int e = 0; e < E; ++e) byu[(size_t)cur[(size_t)g->U[e]]++] = e;
        }
        std::vector<int> cnt((size_t)E, 0);
        std::vector<std::pair<int, int>> tmp;
        std::vector<long long> at((size_t)E, -1);
        for (int u = 0; u < N; ++u) {
            if (first[(size_t)u] == first[(size_t)u + 1]) continue;
            for (int s = off[u]; s < off[u + 1]; ++s) {
                stamp[(size_t)tg[s]] = u;
                slot_of[(size_t)tg[s]] = s;
            }
            for (int q = first[(size_t)u]; q < first[(size_t)u + 1]; ++q) {
                const int e = byu[(size_t)q], v = g->V[e];
                at[(size_t)e] = (long long)tmp.size();
                for (int s = off[v]; s < off[v + 1]; ++s) {
                    const int x = tg[s];
                    if (stamp[(size_t)x] == u) tmp.emplace_back(ei[slot_of[(size_t)x]], ei[s]);
                }
                cnt[(size_t)e] = (int)((long long)tmp.size() - at[(size_t)e]);
            }
        }
        for (int e = 0; e < E; ++e) ioff[(size_t)e + 1] = ioff[(size_t)e] + cnt[(size_t)e];
        pairs.resize(2 * tmp.size());
        for (int e = 0; e < E; ++e)
            for (int k = 0; k < cnt[(size_t)e]; ++k) {
                const auto &pr = tmp[(size_t)(at[(size_t)e] + k)];
                pairs[2 * ((size_t)ioff[(size_t)e] + k)] = pr.first;
                pairs[2 * ((size_t)ioff[(size_t)e] + k) + 1] = pr.second;
            }
        return;
    }
    for (int e = 0; e < E; ++e) {
        int iu = off[g->U[e]], iu_end = off[g->U[e] + 1];
        int iv = off[g->V[e]], iv_end = off[g->V[e] + 1];
        while (iu < iu_end && iv < iv_end) {
            int x = tg[iu], y = tg[iv];
            if (x == y) { pairs.push_back(ei[iu]); pairs.push_back(ei[iv]); }
            iu += (x <= y);
            iv += (x >= y);
        }
        ioff[(size_t)e + 1] = (int)(pairs.size() / 2);
    }
}

namespace {

int lcg15(unsigned int *s)
{
    *s = *s * 1103515245u + 12345u;
    return (int)((*s >> 16) & 0x7fff);
}

// Sampled positions within the stride: n draws of a 62-bit LCG value
// (first draw in the high part) modulo the stride's size, sorted and
// de-duplicated (libdress/src/delta_dress_impl.c:153-157, 234-254).
std::vector<long long> sample_picks(long long per, int n, unsigned int seed, int offset)
{
    long long lim = n < per ? n : per;
    std::vector<long long> p((size_t)lim);
    unsigned int s = seed + (unsigned int)offset;
    for (long long i = 0; i < lim; ++i) {
        long long hi = lcg15(&s);
        long long lo = lcg15(&s);
        p[(size_t)i] = (((hi << 31) | lo) & 0x7FFFFFFFFFFFFFFFLL) % per;
    }
    std::sort(p.begin(), p.end());
    p.erase(std::unique(p.begin(), p.end()), p.end());
    return p;
}

inline int next_pow2(int x)
{
    int m = 1;
    while (m < x) m <<= 1;
    return m;
}

// Everything one request needs, prepared on the host.
struct Prep {
    dressx_hist_request_t *r = nullptr;
    p_dress_graph_t g = nullptr;
    int N = 0, E = 0, S = 0, T = 0;
    long long total = 0;               // C(N,k) or P(N,k)
    long long per = 0;                 // ranks in this stride
    std::vector<long long> ranks;      // sampled ranks (empty = all of the stride)
    long long items = 0;               // subgraphs to process
    bool inplace = false;              // k == 0
    bool empty = false;                // nothing to fit
    bool batchable = false;
    std::vector<int> ioff, pairs;      // common-neighbour pairs (parent numbering)
    int M = 0;
    double *ms_host = nullptr;         // multiset matrix (caller owns after return)
    std::vector<long long> values_host;  // per-subgraph path: values collected on the host
    std::vector<long long> hist;       // flat [bits, count]
    int64_t *hist_mal = nullptr;       // ... or already in a malloc'd array
    long long hist_mal_len = 0;
    unsigned long long sweeps = 0, edge_iters = 0, fits = 0;
};

Status prepare(Prep &p)
{
    dressx_hist_request_t *r = p.r;
    p_dress_graph_t g = r->graph;
    if (!g) return Status::Err(DRESSX_EINVAL, "request without graph");
    if (r->kind != DRESSX_DELTA && r->kind != DRESSX_NABLA) return Status::Err(DRESSX_EINVAL, "bad request kind");
    if (r->stride < 1 || r->offset < 0) return Status::Err(DRESSX_EINVAL, "bad offset/stride");
    p.g = g;
    p.N = g->N;
    p.E = g->E;
    p.S = g->N > 0 ? g->adj_offset[g->N] : 0;
    const int k = r->k;
    p.total = k == 0 ? 1 : (r->kind == DRESSX_DELTA ? binom_h(p.N, k) : perm_h(p.N, k));
    r->num_subgraphs = p.total;
    const bool want_ms = r->keep_multisets != 0;
    // matrices beyond 2^31 entries are not allocated (the caller gets NULL,
    // as when the reference's malloc fails)
    if (want_ms && p.total >= 0 && (p.E == 0 || p.total <= (1LL << 31) / p.E)) {
        size_t len = (size_t)p.total * (size_t)p.E;
        p.ms_host = (double *)std::malloc((len ? len : 1) * sizeof(double));
        if (p.ms_host)
            for (size_t i = 0; i < len; ++i) p.ms_host[i] = std::nan("");
    }
    if (k == 0) {
        p.inplace = r->offset == 0;
        p.empty = !p.inplace;
        return Status::Ok();
    }
    if (k < 0 || k >= p.N) {
        p.empty = true;
        return Status::Ok();
    }
    p.per = (p.total + r->stride - 1 - r->offset) / r->stride;
    if (p.per < 0) p.per = 0;
    if (r->n_samples > 0 && r->n_samples < p.per) {
        std::vector<long long> picks = sample_picks(p.per, r->n_samples, r->seed, r->offset);
        p.ranks.resize(picks.size());
        for (size_t i = 0; i < picks.size(); ++i) p.ranks[i] = r->offset + picks[i] * (long long)r->stride;
        p.items = (long long)picks.size();
    } else {
        p.items = p.per;
    }
    if (p.items == 0) {
        p.empty = true;
        return Status::Ok();
    }

    // common-neighbour pairs of the parent by the reference's merge walk
    // (libdress/src/dress.c:307-363); masks filter them per subgraph
    int maxdeg = 0;
    bool dup = false;
    merge_walk_pairs(g, p.ioff, p.pairs, maxdeg, dup);
    p.T = p.ioff[(size_t)p.E];
    p.M = std::max(2, next_pow2(maxdeg + 1));
    // Masks reproduce the rebuilt subgraph except for the reciprocal-weight
    // lookup of DIRECTED graphs with repeated directed edges.
    // The batch kernel also needs one subgraph's state in shared memory;
    // rows of any length are summed there (certified sums, no networks).
    p.batchable = !(dup && g->variant == DRESS_VARIANT_DIRECTED) &&
                  batch_group_bytes(p.E, p.N, k, 32) <= BATCH_GROUP_BYTES_MAX;
    return Status::Ok();
}

// ---- per-subgraph path ----------------------------------------------------------
Status run_per_fit(Prep &p, const Ctx &ctx)
{
    dressx_hist_request_t *r = p.r;
    p_dress_graph_t g = p.g;
    const int N = p.N, E = p.E, k = r->k;
    std::vector<int> sel((size_t)k);
    std::vector<int> vmap((size_t)N);
    auto process = [&](long long s) -> Status {
        // unrank s
        if (r->kind == DRESSX_DELTA) {
            long long rr = s;
            int c = 0;
            for (int i = 0; i < k; ++i) {
                for (;;) {
                    long long cnt = binom_h(N - c - 1, k - i - 1);
                    if (rr < cnt) break;
                    rr -= cnt;
                    ++c;
                }
                sel[(size_t)i] = c++;
            }
        } else {
            long long rr = s;
            for (int i = 0; i < k; ++i) {
                long long per = perm_h(N - i - 1, k - i - 1);
                long long idx = rr / per;
                rr -= idx * per;
                int v = 0, seen = -1;
                for (;; ++v) {
                    bool used = false;
                    for (int j = 0; j < i; ++j) used |= sel[(size_t)j] == v;
                    if (!used && ++seen == idx) break;
                }
                sel[(size_t)i] = v;
            }
        }
        // build the subgraph (libdress/src/delta_dress_impl.c:33-107,
        // nabla_dress_impl.c:61-91)
        int sN = N, sE = 0;
        int *sU, *sV;
        double *sW = nullptr, *sNW = nullptr;
        std::vector<int> emap((size_t)E, -1);
        if (r->kind == DRESSX_DELTA) {
            int nid = 0;
            for (int v = 0; v < N; ++v) {
                bool del = false;
                for (int i = 0; i < k; ++i) del |= sel[(size_t)i] == v;
                vmap[(size_t)v] = del ? -1 : nid++;
            }
            sN = N - k;
            for (int e = 0; e < E; ++e) sE += vmap[(size_t)g->U[e]] >= 0 && vmap[(size_t)g->V[e]] >= 0;
            if (sE == 0) return Status::Ok();
            sU = (int *)std::malloc((size_t)sE * sizeof(int));
            sV = (int *)std::malloc((size_t)sE * sizeof(int));
            if (g->W) sW = (double *)std::malloc((size_t)sE * sizeof(double));
            for (int e = 0, j = 0; e < E; ++e) {
                int a = vmap[(size_t)g->U[e]], b = vmap[(size_t)g->V[e]];
                if (a >= 0 && b >= 0) {
                    sU[j] = a; sV[j] = b;
                    if (sW) sW[j] = g->W[e];
                    emap[(size_t)e] = j++;
                }
            }
        } else {
            sE = E;
            sU = (int *)std::malloc((size_t)(E ? E : 1) * sizeof(int));
            sV = (int *)std::malloc((size_t)(E ? E : 1) * sizeof(int));
            std::memcpy(sU, g->U, (size_t)E * sizeof(int));
            std::memcpy(sV, g->V, (size_t)E * sizeof(int));
            if (g->W) {
                sW = (double *)std::malloc((size_t)(E ? E : 1) * sizeof(double));
                std::memcpy(sW, g->W, (size_t)E * sizeof(double));
            }
            sNW = (double *)std::malloc((size_t)(N ? N : 1) * sizeof(double));
            for (int v = 0; v < N; ++v) sNW[v] = 1.0;
            static const int pr[16] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53};
            for (int i = 0; i < k; ++i)
                sNW[sel[(size_t)i]] = std::sqrt((double)(i < 16 ? pr[i] : 2 * i + 3));
            for (int e = 0; e < E; ++e) emap[(size_t)e] = e;
        }
        p_dress_graph_t sub = dress_init_graph(sN, sE, sU, sV, sW, sNW, g->variant, g->precompute_intercepts);
        if (!sub) return Status::Err(DRESSX_EINVAL, "subgraph construction failed");
        FitStats fs;
        Status st = fit_graph(sub, r->max_iterations, r->epsilon, nullptr, nullptr, &fs, ctx);
        if (!st.ok()) {
            dress_free_graph(sub);
            return st;
        }
        for (int e = 0; e < sub->E; ++e) {
            long long b;
            std::memcpy(&b, &sub->edge_dress[e], sizeof(b));
            p.values_host.push_back(b);
        }
        if (p.ms_host)
            for (int e = 0; e < E; ++e)
                p.ms_host[(size_t)s * E + e] = emap[(size_t)e] >= 0 ? sub->edge_dress[emap[(size_t)e]] : std::nan("");
        p.sweeps += (unsigned long long)fs.sweeps;
        p.edge_iters += (unsigned long long)fs.sweeps * (unsigned long long)sub->E;
        p.fits += 1;
        dress_free_graph(sub);
        return Status::Ok();
    };
    for (long long i = 0; i < p.items; ++i) {
        long long s = p.ranks.empty() ? r->offset + i * (long long)r->stride : p.ranks[(size_t)i];
        DRESS_TRY(process(s));
    }
    return Status::Ok();
}

// ---- histogram of host-collected values (in-place fits, per-subgraph path) -------
Status hist_of_host_values(std::vector<Prep *> &ps, cudaStream_t st, int sms)
{
    long long total = 0;
    for (Prep *p : ps) total += (long long)p->values_host.size();
    if (total == 0) return Status::Ok();
    DevBuf<unsigned long long> keys, alt;
    DRESS_TRY(keys.alloc((size_t)total, st));
    DRESS_TRY(alt.alloc((size_t)total, st));
    std::vector<long long> begin, len;
    long long o = 0;
    for (Prep *p : ps) {
        begin.push_back(o);
        len.push_back((long long)p->values_host.size());
        if (!p->values_host.empty())
            DRESS_CUDA_TRY(counted_memcpy(keys.get() + o, p->values_host.data(),
                                           p->values_host.size() * sizeof(long long), cudaMemcpyHostToDevice, st));
        o += (long long)p->values_host.size();
    }
    std::vector<std::vector<long long>> out;
    DRESS_TRY(histogram_segments(keys.get(), alt.get(), begin, len, out, st, sms));
    for (size_t i = 0; i < ps.size(); ++i) ps[i]->hist = std::move(out[i]);
    return Status::Ok();
}

// ---- batched path ------------------------------------------------------------------
struct Tune {
    int gsize, groups;
    int per_sm = 1;          // CTAs meant to share an SM (shared memory split between them)
};

// Threads per subgraph by edge count (sweeps of a few hundred edges keep a
// warp busy; larger subgraphs split across more warps), unless the autotuner
// has measured this size class.
struct TuneKey {
    int e, n, M, k;
    bool operator<(const TuneKey &o) const
    {
        return e != o.e ? e < o.e : n != o.n ? n < o.n : M != o.M ? M < o.M : k < o.k;
    }
};
std::mutex g_tuned_mu;
std::map<TuneKey, Tune> g_tuned;    // size class -> measured best schedule

TuneKey tune_key(int maxE, int maxN, int M, int maxk)
{
    return {next_pow2(maxE), next_pow2(maxN), M, maxk};
}

Tune pick_tune(int maxE, int maxN, int M, int maxk, const dressx_config_t &cfg)
{
    int gs = cfg.group_threads > 0 ? cfg.group_threads
           : maxE <= 640 ? 32 : maxE <= 2048 ? 64 : maxE <= 8192 ? 128 : 256;
    if (cfg.group_threads <= 0) {
        std::lock_guard<std::mutex> lk(g_tuned_mu);
        auto it = g_tuned.find(tune_key(maxE, maxN, M, maxk));
        if (it != g_tuned.end()) return it->second;
    }
    int groups = 512 / gs;
    if (gs > 32 && groups > 15) groups = 15;
    return {gs, groups, 1};
}

// Groups per CTA and parent staging for a given group size: as many groups
// as shared memory holds (at most `groups`), staging the parent unless that
// halves the groups.  False when not even one group fits.
bool shape_launch(BatchLaunch &L, const Tune &tu, long long smem_cap_full, long long smem_sm = 0)
{
    // two CTAs per SM split the SM's shared memory (each keeps ~1 KB of
    // system and static shared memory)
    const long long smem_cap = tu.per_sm == 2 && smem_sm > 0 ? smem_sm / 2 - 2048 : smem_cap_full;
    L.min_ctas = tu.per_sm == 2 && smem_sm > 0 ? 2 : 1;
    L.gsize = tu.gsize;
    L.per_group = 0;
    L.stage = 1;
    L.groups = tu.groups;
    while (L.groups > 1 && (long long)batch_smem_bytes(L) > smem_cap) --L.groups;
    if ((long long)batch_smem_bytes(L) > smem_cap) {
        L.stage = 0;
        L.groups = tu.groups;
        while (L.groups > 1 && (long long)batch_smem_bytes(L) > smem_cap) --L.groups;
    }
    if ((long long)batch_smem_bytes(L) > smem_cap) return false;
    if (L.stage && L.groups * 2 < tu.groups) {
        // staging leaves too few groups: read parents from L2 instead
        BatchLaunch L2 = L;
        L2.stage = 0;
        L2.groups = tu.groups;
        while (L2.groups > 1 && (long long)batch_smem_bytes(L2) > smem_cap) --L2.groups;
        if (L2.groups > L.groups) L = L2;
    }
    return true;
}

// Chunks: a few rounds of subgraphs per CTA visit, requests in order; with
// limit >= 0 only the first `limit` subgraphs of the whole batch.
void build_chunks(const std::vector<Prep *> &ps, int groups, long long limit, std::vector<Chunk> &chunks)
{
    chunks.clear();
    const int chunk_items = 4 * groups;
    long long taken = 0;
    for (size_t i = 0; i < ps.size(); ++i)
        for (long long f = 0; f < ps[i]->items; f += chunk_items) {
            if (limit >= 0 && taken >= limit) return;
            int c = (int)std::min<long long>(chunk_items, ps[i]->items - f);
            chunks.push_back({(int)i, c, f});
            taken += c;
        }
}

// A packed, uploaded batch: parents, chunks, value and statistics buffers.
struct BatchPlan {
    std::vector<Prep *> ps;
    BatchLaunch L{};
    std::vector<ParentDesc> descs;
    std::vector<Chunk> chunks;
    std::vector<long long> val_base;
    long long values = 0, ms_total = 0;
    DevBuf<unsigned char> d_pdata;
    DevBuf<ParentDesc> d_desc;
    DevBuf<Chunk> d_chunks;
    DevBuf<long long> d_ranks;
    DevBuf<unsigned long long> d_vals, d_alt, d_stats;
    DevBuf<double> d_ms;
    DevBuf<int> d_counter;
    std::vector<unsigned long long> stats;
    HistResult hist;
    bool need_hist = false;
    float fit_ms = 0.f, hist_ms = 0.f;       // device time of the last run
    long long smem_cap = 0, smem_sm = 0;
    int tuned_per_sm = 1;                    // CTAs per SM the autotuner chose
    cudaGraphExec_t gexec = nullptr;         // captured fit stage (dressx_batch_capture)
    ~BatchPlan()
    {
        if (gexec) cudaGraphExecDestroy(gexec);
    }
};

Status plan_batched(std::vector<Prep *> &ps, const Ctx &en, BatchPlan &P)
{
    P.ps = ps;
    cudaStream_t st = en.st;
    int smem_optin = 0;
    DRESS_CUDA_TRY(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, en.device));
    const long long smem_cap = smem_optin - 256;

    // one launch for all batchable requests
    int maxE = 1, maxN = 1, maxk = 1, M = 2;
    long long maxbytes = 16, arena = 0, values = 0, ms_total = 0, nranks = 0;
    std::vector<ParentDesc> &descs = P.descs;
    std::vector<long long> &val_base = P.val_base;
    // byte / element offsets of each request's sections, turned into device
    // pointers once the buffers exist
    std::vector<long long> data_off, ranks_off, ms_off;
    for (Prep *p : ps) {
        ParentLayout PL = parent_layout(p->N, p->E, p->S, p->T, 0, 0);
        maxE = std::max(maxE, p->E);
        maxN = std::max(maxN, p->N);
        maxk = std::max(maxk, p->r->k);
        M = std::max(M, p->M);
        maxbytes = std::max(maxbytes, PL.bytes);
        ParentDesc d{};
        d.N = p->N; d.E = p->E; d.S = p->S; d.T = p->T;
        d.kind = p->r->kind == DRESSX_DELTA ? ITEM_DELTA : ITEM_NABLA;
        d.k = p->r->k;
        d.fwd = p->g->variant == DRESS_VARIANT_FORWARD || p->g->variant == DRESS_VARIANT_BACKWARD;
        d.force_exact = en.cfg->exact_sums != 0;
        d.max_iter = p->r->max_iterations;
        d.eps = p->r->epsilon;
        d.offset = p->r->offset;
        d.stride = p->r->stride;
        data_off.push_back(arena);
        ranks_off.push_back(p->ranks.empty() ? -1 : nranks);
        ms_off.push_back(p->ms_host ? ms_total : -1);
        descs.push_back(d);
        val_base.push_back(values);
        arena += PL.bytes;
        values += p->items * (long long)p->E;
        nranks += (long long)p->ranks.size();
        if (p->ms_host) ms_total += p->total * (long long)p->E;
    }
    Tune tu = pick_tune(maxE, maxN, M, maxk, *en.cfg);
    BatchLaunch &L = P.L;
    L.maxE = maxE;
    L.maxN = maxN;
    L.maxk = maxk;
    L.M = M;
    L.parent_bytes = maxbytes;
    P.smem_cap = smem_cap;
    int smem_sm = 0;
    DRESS_CUDA_TRY(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, en.device));
    P.smem_sm = smem_sm;
    if (!shape_launch(L, tu, smem_cap, smem_sm))
        return Status::Err(DRESSX_EUNSUPPORTED, "subgraph state exceeds shared memory");

    // pack parents, several threads for many, into the pinned stage when it
    // can hold them (the upload is then one DMA; the stage is free again
    // when this function returns)
    unsigned char *hbytes = nullptr;
    std::unique_ptr<unsigned char[]> hheap;
    const bool staged = en.stage && en.stage->reserve((size_t)arena).ok();
    if (staged) {
        hbytes = (unsigned char *)en.stage->ptr();
    } else {
        hheap.reset(new unsigned char[(size_t)arena]);
        hbytes = hheap.get();
    }
    std::vector<long long> hranks((size_t)nranks);
    parallel_for((long long)ps.size(), host_threads((long long)ps.size() / 16), [&](long long ii) {
        const size_t i = (size_t)ii;
        Prep *p = ps[i];
        p_dress_graph_t g = p->g;
        ParentLayout PL = parent_layout(p->N, p->E, p->S, p->T, 0, 0);
        unsigned char *b = hbytes + data_off[i];
        std::memcpy(b + PL.U, g->U, (size_t)p->E * 4);
        std::memcpy(b + PL.V, g->V, (size_t)p->E * 4);
        std::memcpy(b + PL.w, g->edge_weight, (size_t)p->E * 8);
        std::memcpy(b + PL.row_off, g->adj_offset, (size_t)(p->N + 1) * 4);
        std::memcpy(b + PL.row_eid, g->adj_edge_idx, (size_t)p->S * 4);
        std::memcpy(b + PL.ioff, p->ioff.data(), (size_t)(p->E + 1) * 4);
        if (p->T) std::memcpy(b + PL.pairs, p->pairs.data(), (size_t)p->T * 8);
        if (!p->ranks.empty()) std::copy(p->ranks.begin(), p->ranks.end(), hranks.begin() + ranks_off[i]);
    }, 16);
    std::vector<Chunk> &chunks = P.chunks;
    build_chunks(ps, L.groups, -1, chunks);

    const int nreq = (int)ps.size();
    DevBuf<unsigned char> &d_pdata = P.d_pdata;
    DevBuf<ParentDesc> &d_desc = P.d_desc;
    DevBuf<Chunk> &d_chunks = P.d_chunks;
    DevBuf<long long> &d_ranks = P.d_ranks;
    DevBuf<unsigned long long> &d_vals = P.d_vals, &d_stats = P.d_stats;
    DevBuf<double> &d_ms = P.d_ms;
    DevBuf<int> &d_counter = P.d_counter;
    P.values = values;
    P.ms_total = ms_total;
    DRESS_TRY(d_pdata.alloc((size_t)arena, st));
    DRESS_TRY(d_desc.alloc(descs.size(), st));
    DRESS_TRY(d_chunks.alloc(chunks.size(), st));
    DRESS_TRY(d_ranks.alloc(hranks.size() + 1, st));
    DRESS_TRY(d_vals.alloc((size_t)values + 1, st));
    DRESS_TRY(d_stats.alloc(ST_WORDS * (size_t)nreq, st));
    DRESS_TRY(d_counter.alloc(1, st));
    if (ms_total > 0) DRESS_TRY(d_ms.alloc((size_t)ms_total, st));
    for (int i = 0; i < nreq; ++i) {
        ParentDesc &d = descs[(size_t)i];
        d.data = d_pdata.get() + data_off[(size_t)i];
        d.values = (double *)d_vals.get() + val_base[(size_t)i];
        d.stats = d_stats.get() + ST_WORDS * (size_t)i;
        d.multisets = ms_off[(size_t)i] >= 0 ? d_ms.get() + ms_off[(size_t)i] : nullptr;
        d.ranks = ranks_off[(size_t)i] >= 0 ? d_ranks.get() + ranks_off[(size_t)i] : nullptr;
    }
    DRESS_CUDA_TRY(counted_memcpy(d_pdata.get(), hbytes, (size_t)arena, cudaMemcpyHostToDevice, st));
    DRESS_CUDA_TRY(counted_memcpy(d_desc.get(), descs.data(), descs.size() * sizeof(ParentDesc),
                                   cudaMemcpyHostToDevice, st));
    DRESS_CUDA_TRY(counted_memcpy(d_chunks.get(), chunks.data(), chunks.size() * sizeof(Chunk),
                                   cudaMemcpyHostToDevice, st));
    if (!hranks.empty())
        DRESS_CUDA_TRY(counted_memcpy(d_ranks.get(), hranks.data(), hranks.size() * sizeof(long long),
                                       cudaMemcpyHostToDevice, st));
    if (ms_total > 0) {
        // the rows of unprocessed subgraphs stay NaN, as in the reference
        size_t o = 0;
        for (Prep *p : ps)
            if (p->ms_host) {
                size_t len = (size_t)p->total * (size_t)p->E;
                DRESS_CUDA_TRY(counted_memcpy(d_ms.get() + o, p->ms_host, len * sizeof(double),
                                               cudaMemcpyHostToDevice, st));
                o += len;
            }
    }
    L.parents = d_desc.get();
    L.chunks = d_chunks.get();
    L.nchunks = (int)chunks.size();
    L.chunk_counter = d_counter.get();
    L.per_group = 0;
    P.need_hist = false;
    for (Prep *p : ps) P.need_hist |= p->r->want_histogram != 0;
    if (P.need_hist) DRESS_TRY(P.d_alt.alloc((size_t)values + 1, st));
    if (staged) DRESS_CUDA_TRY(cudaStreamSynchronize(st));
    return Status::Ok();
}

// Device work of a planned batch: all fits, then the histograms (left in
// device memory).  Can be repeated; each run starts from the same inputs.
// The fit stage: counters reset and the batch kernel.  It allocates nothing
// and never synchronises, so it can be captured into a CUDA graph.
Status enqueue_fit(BatchPlan &P, cudaStream_t st, int sms)
{
    const int nreq = (int)P.ps.size();
    DRESS_CUDA_TRY(cudaMemsetAsync(P.d_stats.get(), 0, ST_WORDS * (size_t)nreq * sizeof(unsigned long long), st));
    DRESS_CUDA_TRY(cudaMemsetAsync(P.d_counter.get(), 0, sizeof(int), st));
    return launch_batch(P.L, sms, st);
}

Status exec_batched(BatchPlan &P, const Ctx &en)
{
    cudaStream_t st = en.st;
    const int nreq = (int)P.ps.size();
    cudaEvent_t ev[3];
    for (auto &e : ev) DRESS_CUDA_TRY(cudaEventCreate(&e));
    DRESS_CUDA_TRY(cudaEventRecord(ev[0], st));
    if (P.gexec) {
        count_launch();
        DRESS_CUDA_TRY(cudaGraphLaunch(P.gexec, st));
    } else {
        DRESS_TRY(enqueue_fit(P, st, en.num_sms));
    }
    DRESS_CUDA_TRY(cudaEventRecord(ev[1], st));
    P.stats.assign(ST_WORDS * (size_t)nreq, 0);
    DRESS_CUDA_TRY(counted_memcpy(P.stats.data(), P.d_stats.get(), P.stats.size() * sizeof(unsigned long long),
                                   cudaMemcpyDeviceToHost, st));
    DRESS_CUDA_TRY(cudaStreamSynchronize(st));
    if (P.need_hist) {
        std::vector<long long> begin((size_t)nreq), len((size_t)nreq);
        for (int i = 0; i < nreq; ++i) {
            begin[(size_t)i] = P.val_base[(size_t)i];
            len[(size_t)i] = (long long)P.stats[ST_WORDS * (size_t)i + ST_CURSOR];
        }
        DRESS_TRY(histogram_device(P.d_vals.get(), P.d_alt.get(), begin, len, P.hist, st, en.num_sms));
    }
    DRESS_CUDA_TRY(cudaEventRecord(ev[2], st));
    DRESS_CUDA_TRY(cudaStreamSynchronize(st));
    cudaEventElapsedTime(&P.fit_ms, ev[0], ev[1]);
    cudaEventElapsedTime(&P.hist_ms, ev[1], ev[2]);
    for (auto &e : ev) cudaEventDestroy(e);
    return Status::Ok();
}

// Results of the last run into the requests' host-side state.
// pre/cap (nullable): host arrays already allocated per request, with
// their capacity in int64 words; the histograms that fit go there (their
// ownership passes to the request, the entry is cleared).
Status collect_batched(BatchPlan &P, const Ctx &en, std::vector<int64_t *> *pre = nullptr,
                       const std::vector<long long> *cap = nullptr)
{
    cudaStream_t st = en.st;
    const int nreq = (int)P.ps.size();
    std::vector<Prep *> &ps = P.ps;
    for (int i = 0; i < nreq; ++i) {
        const unsigned long long *st_i = P.stats.data() + ST_WORDS * (size_t)i;
        ps[(size_t)i]->sweeps = st_i[ST_SWEEPS];
        ps[(size_t)i]->edge_iters = st_i[ST_EDGE_ITERS];
        ps[(size_t)i]->fits = st_i[ST_FITS];
    }
    if (P.need_hist) {
        std::vector<int64_t *> outs;
        std::vector<long long> lens;
        DRESS_TRY(histogram_fetch(P.hist, outs, lens, en.stage, st, en.num_sms, pre, cap));
        for (int i = 0; i < nreq; ++i) {
            std::free(ps[(size_t)i]->hist_mal);
            ps[(size_t)i]->hist_mal = outs[(size_t)i];
            ps[(size_t)i]->hist_mal_len = lens[(size_t)i];
        }
    }
    if (P.ms_total > 0) {
        size_t o = 0;
        for (Prep *p : ps)
            if (p->ms_host) {
                size_t n = (size_t)p->total * (size_t)p->E;
                DRESS_CUDA_TRY(counted_memcpy(p->ms_host, P.d_ms.get() + o, n * sizeof(double),
                                               cudaMemcpyDeviceToHost, st));
                o += n;
            }
        DRESS_CUDA_TRY(cudaStreamSynchronize(st));
    }
    return Status::Ok();
}

// Autotuner: times the fit stage on the first subgraphs of the batch for
// every group size whose state fits shared memory, records the fastest for
// this size class (later batches of the class are planned with it) and
// re-plans this batch with it.
Status autotune_batched(BatchPlan &P, const Ctx &en, int *best_out, std::vector<float> *rates)
{
    cudaStream_t st = en.st;
    long long total = 0;
    for (Prep *p : P.ps) total += p->items;
    if (total == 0) return Status::Ok();
    // the whole batch up to 200K subgraphs (a sample leaves too few chunks per
    // SM to show the tail of a schedule), a spread quarter beyond
    const long long limit = total <= 200000 ? total : std::max<long long>(200000, total / 4);
    struct Cand { int gs, per_sm; };
    std::vector<Cand> cands = {{32, 1}, {64, 1}, {128, 1}, {256, 1}, {32, 2}, {64, 2}, {128, 2}};
    DevBuf<Chunk> d_try;
    cudaEvent_t e0, e1;
    DRESS_CUDA_TRY(cudaEventCreate(&e0));
    DRESS_CUDA_TRY(cudaEventCreate(&e1));
    int best = -1;
    double best_rate = 0.0;
    Status err;
    Tune best_tu{0, 0, 1};
    std::vector<std::pair<double, Tune>> tried;
    for (const Cand &cd : cands) {
        const int gs = cd.gs;
        Tune tu{gs, gs == 32 ? 16 : std::min(15, 512 / gs), cd.per_sm};
        BatchLaunch L = P.L;
        if (!shape_launch(L, tu, P.smem_cap, P.smem_sm)) {
            if (rates) rates->push_back(0.f);
            continue;
        }
        // a sample spread over the whole batch: every k-th chunk
        std::vector<Chunk> all, ch;
        build_chunks(P.ps, L.groups, -1, all);
        const long long k = std::max<long long>(1, (total + limit - 1) / limit);
        for (size_t c = 0; c < all.size(); c += (size_t)k) ch.push_back(all[c]);
        long long items = 0;
        for (const Chunk &c : ch) items += c.count;
        err = d_try.alloc(ch.size(), st);
        if (!err.ok()) break;
        if (cudaMemcpyAsync(d_try.get(), ch.data(), ch.size() * sizeof(Chunk), cudaMemcpyHostToDevice, st) != cudaSuccess) {
            err = Status::Err(DRESSX_ECUDA, "autotune: chunk upload failed");
            break;
        }
        L.chunks = d_try.get();
        L.nchunks = (int)ch.size();
        float ms = 0.f;
        std::vector<float> times;
        for (int rep = 0; rep < 4; ++rep) {          // the first run is untimed; the median of three
            cudaMemsetAsync(P.d_stats.get(), 0, ST_WORDS * P.ps.size() * sizeof(unsigned long long), st);
            cudaMemsetAsync(P.d_counter.get(), 0, sizeof(int), st);
            cudaEventRecord(e0, st);
            err = launch_batch(L, en.num_sms, st);
            if (!err.ok()) break;
            cudaEventRecord(e1, st);
            if (cudaStreamSynchronize(st) != cudaSuccess) {
                err = Status::Err(DRESSX_ECUDA, "autotune: run failed");
                break;
            }
            cudaEventElapsedTime(&ms, e0, e1);
            if (rep > 0) times.push_back(ms);
        }
        if (!err.ok()) break;
        std::sort(times.begin(), times.end());
        const float med = times.empty() ? 0.f : times[times.size() / 2];
        const double rate = med > 0.f ? (double)items / med : 0.0;
        if (rates) rates->push_back((float)rate);
        tried.push_back({rate, tu});
        best_rate = std::max(best_rate, rate);
    }
    // The first candidate, in the fixed order above, within 3 % of the
    // fastest: schedules that differ by less than the run-to-run noise then
    // resolve the same way on every run.
    for (const auto &t : tried)
        if (t.first > 0.0 && t.first >= 0.97 * best_rate) {
            best = t.second.gsize;
            best_tu = t.second;
            break;
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    DRESS_TRY(err);
    if (best < 0) return Status::Err(DRESSX_EUNSUPPORTED, "autotune: no group size fits");
    {
        std::lock_guard<std::mutex> lk(g_tuned_mu);
        g_tuned[tune_key(P.L.maxE, P.L.maxN, P.L.M, P.L.maxk)] = best_tu;
    }
    if (!shape_launch(P.L, best_tu, P.smem_cap, P.smem_sm))
        return Status::Err(DRESSX_EUNSUPPORTED, "autotune: re-plan failed");
    P.tuned_per_sm = best_tu.per_sm;
    build_chunks(P.ps, P.L.groups, -1, P.chunks);
    DRESS_TRY(P.d_chunks.alloc(P.chunks.size(), st));
    DRESS_CUDA_TRY(counted_memcpy(P.d_chunks.get(), P.chunks.data(), P.chunks.size() * sizeof(Chunk),
                                   cudaMemcpyHostToDevice, st));
    P.L.chunks = P.d_chunks.get();
    P.L.nchunks = (int)P.chunks.size();
    if (P.gexec) {                       // the captured stage has the old schedule
        cudaGraphExecDestroy(P.gexec);
        P.gexec = nullptr;
    }
    DRESS_CUDA_TRY(cudaStreamSynchronize(st));
    if (best_out) *best_out = best;
    return Status::Ok();
}

// Captures the fit stage into a CUDA graph that exec_batched replays.
Status capture_batched(BatchPlan &P, const Ctx &en)
{
    if (P.gexec) {
        cudaGraphExecDestroy(P.gexec);
        P.gexec = nullptr;
    }
    DRESS_CUDA_TRY(cudaStreamSynchronize(en.st));
    cudaGraph_t g = nullptr;
    DRESS_CUDA_TRY(cudaStreamBeginCapture(en.st, cudaStreamCaptureModeThreadLocal));
    Status s = enqueue_fit(P, en.st, en.num_sms);
    cudaError_t e = cudaStreamEndCapture(en.st, &g);
    if (!s.ok() || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        return s.ok() ? Status::Err(DRESSX_ECUDA, std::string("stream capture: ") + cudaGetErrorString(e)) : s;
    }
    e = cudaGraphInstantiate(&P.gexec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        P.gexec = nullptr;
        return Status::Err(DRESSX_ECUDA, std::string("graph instantiation: ") + cudaGetErrorString(e));
    }
    return Status::Ok();
}

// Host arrays for the histograms, allocated while the fits run.  A request's
// histogram has at most one pair per value, and it has at most subgraphs x
// edges values, so arrays of that size are allocated and their pages mapped
// (a write to each page) by host threads during the device work; the fetch
// then only copies, and trims each array to its length.  Only when the
// bounds add up to a moderate size.
constexpr long long PREFAULT_MIN_BYTES = 64LL << 20;
constexpr long long PREFAULT_MAX_BYTES = 4LL << 30;

struct Prefault {
    std::vector<int64_t *> arr;
    std::vector<long long> cap;          // int64 words
    std::vector<std::thread> th;
    void start(const std::vector<Prep *> &ps)
    {
        long long total = 0;
        cap.assign(ps.size(), 0);
        for (size_t i = 0; i < ps.size(); ++i)
            if (ps[i]->r->want_histogram) {
                cap[i] = 2 * ps[i]->items * (long long)ps[i]->E;
                total += cap[i] * 8;
            }
        arr.assign(ps.size(), nullptr);
        if (total < PREFAULT_MIN_BYTES || total > PREFAULT_MAX_BYTES) return;
        // leave a core to the thread that drives the device
        const int nthr = std::max(1, host_threads((long long)ps.size()) - 1);
        for (int t = 0; t < nthr; ++t)
            th.emplace_back([this, t, nthr] {
                for (size_t i = (size_t)t; i < cap.size(); i += (size_t)nthr) {
                    if (!cap[i]) continue;
                    const size_t n = (size_t)cap[i] * sizeof(int64_t);
                    char *a = (char *)std::malloc(n);
                    if (a)
                        for (size_t o = 0; o < n; o += 4096) ((volatile char *)a)[o] = 0;
                    arr[i] = (int64_t *)a;
                }
            });
    }
    void join()
    {
        for (auto &t : th) t.join();
        th.clear();
    }
    ~Prefault()
    {
        join();
        for (int64_t *a : arr) std::free(a);
    }
};

Status run_batched(std::vector<Prep *> &ps, const Ctx &en)
{
    BatchPlan P;
    DRESS_TRY(plan_batched(ps, en, P));
    Prefault pf;
    pf.start(ps);
    Status s = exec_batched(P, en);
    pf.join();
    DRESS_TRY(s);
    return collect_batched(P, en, pf.arr.empty() ? nullptr : &pf.arr, &pf.cap);
}

Status finish(Prep &p)
{
    dressx_hist_request_t *r = p.r;
    r->fits = (int64_t)p.fits;
    r->hist_flat = nullptr;
    r->hist_len = 0;
    if (r->want_histogram && p.hist_mal) {          // hand over the fetched array
        r->hist_flat = p.hist_mal;
        r->hist_len = (int)p.hist_mal_len;
        p.hist_mal = nullptr;
        p.hist_mal_len = 0;
    } else if (r->want_histogram && !p.hist.empty()) {
        r->hist_flat = (int64_t *)std::malloc(p.hist.size() * sizeof(int64_t));
        if (!r->hist_flat) return Status::Err(DRESSX_ENOMEM, "host allocation of the histogram failed");
        std::memcpy(r->hist_flat, p.hist.data(), p.hist.size() * sizeof(int64_t));
        r->hist_len = (int)p.hist.size();
    }
    r->multisets = p.ms_host;
    p.ms_host = nullptr;
    return Status::Ok();
}

}  // namespace

// All requests on one execution context (no locking: the caller owns ctx).
Status hist_batch_core(dressx_hist_request_t *reqs, int n, bool per_fit, const Ctx &ctx, int64_t *edge_sweeps)
{
    DRESS_CUDA_TRY(cudaSetDevice(ctx.device));
    std::vector<Prep> ps((size_t)n);
    std::vector<Status> pst((size_t)n);
    // requests are prepared independently, several threads for many
    parallel_for(n, host_threads(n / 8), [&](long long ii) {
        const size_t i = (size_t)ii;
        ps[i].r = &reqs[i];
        reqs[i].status = DRESSX_OK;
        reqs[i].hist_flat = nullptr;
        reqs[i].hist_len = 0;
        reqs[i].multisets = nullptr;
        reqs[i].fits = 0;
        pst[i] = prepare(ps[i]);
    }, 8);
    Status first;
    for (int i = 0; i < n; ++i) {
        const Status &s = pst[(size_t)i];
        if (!s.ok()) {
            reqs[i].status = s.code;
            if (first.ok()) first = s;
        }
    }
    std::vector<Prep *> batch, host_vals;
    for (auto &p : ps) {
        if (p.r->status != DRESSX_OK || p.empty) continue;
        if (p.inplace) {
            // k == 0: fit the caller's graph itself (libdress/src/delta_dress_impl.c:206-224)
            FitStats fs;
            Status s = fit_graph(p.g, p.r->max_iterations, p.r->epsilon, nullptr, nullptr, &fs, ctx);
            if (!s.ok()) { p.r->status = s.code; if (first.ok()) first = s; continue; }
            for (int e = 0; e < p.E; ++e) {
                long long b;
                std::memcpy(&b, &p.g->edge_dress[e], sizeof(b));
                p.values_host.push_back(b);
                if (p.ms_host) p.ms_host[e] = p.g->edge_dress[e];
            }
            p.fits = 1;
            p.sweeps = (unsigned long long)fs.sweeps;
            p.edge_iters = (unsigned long long)fs.sweeps * (unsigned long long)p.E;
            host_vals.push_back(&p);
        } else if (p.batchable && !per_fit) {
            batch.push_back(&p);
        } else {
            Status s = run_per_fit(p, ctx);
            if (!s.ok()) { p.r->status = s.code; if (first.ok()) first = s; continue; }
            host_vals.push_back(&p);
        }
    }
    if (!batch.empty()) {
        Status s = run_batched(batch, ctx);
        if (!s.ok()) {
            for (Prep *p : batch) p->r->status = s.code;
            if (first.ok()) first = s;
        }
    }
    {
        std::vector<Prep *> hv;
        for (Prep *p : host_vals)
            if (p->r->want_histogram) hv.push_back(p);
        Status s = hist_of_host_values(hv, ctx.st, ctx.num_sms);
        if (!s.ok()) {
            for (Prep *p : hv) p->r->status = s.code;
            if (first.ok()) first = s;
        }
    }
    for (auto &p : ps) {
        if (p.r->status == DRESSX_OK) {
            Status s = finish(p);
            if (!s.ok()) { p.r->status = s.code; if (first.ok()) first = s; }
        }
        if (p.ms_host) { std::free(p.ms_host); p.ms_host = nullptr; }
        std::free(p.hist_mal);
        p.hist_mal = nullptr;
    }
    if (edge_sweeps)
        for (int i = 0; i < n; ++i) edge_sweeps[i] = (int64_t)ps[(size_t)i].edge_iters;
    return first;
}

namespace {

Status hist_batch_impl(dressx_hist_request_t *reqs, int n, bool per_fit)
{
    Engine &en = engine();
    std::lock_guard<std::mutex> lk(en.mu);
    DRESS_TRY(en.init());
    return hist_batch_core(reqs, n, per_fit, en.ctx);
}

// ---- legacy wrappers -------------------------------------------------------------------
int64_t *legacy_flat(int kind, p_dress_graph_t g, int k, int iterations, double epsilon, int n_samples,
                     unsigned int seed, int *hist_size, int keep_multisets, double **multisets,
                     int64_t *num, int offset, int stride)
{
    dressx_hist_request_t r{};
    r.graph = g;
    r.kind = kind;
    r.k = k;
    r.max_iterations = iterations;
    r.epsilon = epsilon;
    r.n_samples = n_samples;
    r.seed = seed;
    r.offset = offset;
    r.stride = stride;
    r.want_histogram = hist_size != nullptr;
    r.keep_multisets = keep_multisets && multisets;
    Status s = hist_batch_impl(&r, 1, false);
    set_last_error(s);
    if (hist_size) *hist_size = 0;
    if (!s.ok()) return nullptr;
    if (num) *num = r.num_subgraphs;
    if (keep_multisets && multisets) *multisets = r.multisets;
    if (hist_size) *hist_size = r.hist_len;
    return r.hist_flat;
}

dress_hist_pair_t *flat_to_pairs(int64_t *flat, int flat_len, int *hist_size)
{
    int n = flat_len / 2;
    if (hist_size) *hist_size = n;
    if (!flat || n <= 0) {
        std::free(flat);
        return nullptr;
    }
    dress_hist_pair_t *pairs = (dress_hist_pair_t *)std::malloc((size_t)n * sizeof(dress_hist_pair_t));
    if (pairs)
        for (int i = 0; i < n; ++i) {
            std::memcpy(&pairs[i].value, &flat[2 * i], sizeof(double));
            pairs[i].count = flat[2 * i + 1];
        }
    std::free(flat);
    return pairs;
}

}  // namespace
}  // namespace dress

using namespace dress;

extern "C" {

int dressx_hist_batch(dressx_hist_request_t *reqs, int n)
{
    if (!reqs || n < 0) return DRESSX_EINVAL;
    Status s = hist_batch_impl(reqs, n, false);
    set_last_error(s);
    return s.code;
}

int dressx_hist_batch_per_fit(dressx_hist_request_t *reqs, int n)
{
    if (!reqs || n < 0) return DRESSX_EINVAL;
    Status s = hist_batch_impl(reqs, n, true);
    set_last_error(s);
    return s.code;
}

int64_t *dress_delta_fit_cuda_strided_flat(p_dress_graph_t g, int k, int iterations, double epsilon, int n_samples,
                                           unsigned int seed, int *hist_size, int keep_multisets,
                                           double **multisets, int64_t *num_subgraphs, int offset, int stride)
{
    return legacy_flat(DRESSX_DELTA, g, k, iterations, epsilon, n_samples, seed, hist_size, keep_multisets,
                       multisets, num_subgraphs, offset, stride);
}

int64_t *dress_delta_fit_cuda_flat(p_dress_graph_t g, int k, int iterations, double epsilon, int n_samples,
                                   unsigned int seed, int *hist_size, int keep_multisets, double **multisets,
                                   int64_t *num_subgraphs)
{
    return legacy_flat(DRESSX_DELTA, g, k, iterations, epsilon, n_samples, seed, hist_size, keep_multisets,
                       multisets, num_subgraphs, 0, 1);
}

dress_hist_pair_t *dress_delta_fit_cuda_strided(p_dress_graph_t g, int k, int iterations, double epsilon,
                                                int n_samples, unsigned int seed, int *hist_size,
                                                int keep_multisets, double **multisets, int64_t *num_subgraphs,
                                                int offset, int stride)
{
    int flat_len = 0;
    int64_t *flat = legacy_flat(DRESSX_DELTA, g, k, iterations, epsilon, n_samples, seed,
                                hist_size ? &flat_len : nullptr, keep_multisets, multisets, num_subgraphs,
                                offset, stride);
    return flat_to_pairs(flat, flat_len, hist_size);
}

dress_hist_pair_t *dress_delta_fit_cuda(p_dress_graph_t g, int k, int iterations, double epsilon, int n_samples,
                                        unsigned int seed, int *hist_size, int keep_multisets,
                                        double **multisets, int64_t *num_subgraphs)
{
    return dress_delta_fit_cuda_strided(g, k, iterations, epsilon, n_samples, seed, hist_size, keep_multisets,
                                        multisets, num_subgraphs, 0, 1);
}

int64_t *dress_nabla_fit_cuda_strided_flat(p_dress_graph_t g, int k, int iterations, double epsilon, int n_samples,
                                           unsigned int seed, int *hist_size, int keep_multisets,
                                           double **multisets, int64_t *num_tuples, int offset, int stride)
{
    return legacy_flat(DRESSX_NABLA, g, k, iterations, epsilon, n_samples, seed, hist_size, keep_multisets,
                       multisets, num_tuples, offset, stride);
}

int64_t *dress_nabla_fit_cuda_flat(p_dress_graph_t g, int k, int iterations, double epsilon, int n_samples,
                                   unsigned int seed, int *hist_size, int keep_multisets, double **multisets,
                                   int64_t *num_tuples)
{
    return legacy_flat(DRESSX_NABLA, g, k, iterations, epsilon, n_samples, seed, hist_size, keep_multisets,
                       multisets, num_tuples, 0, 1);
}

dress_hist_pair_t *dress_nabla_fit_cuda_strided(p_dress_graph_t g, int k, int iterations, double epsilon,
                                                int n_samples, unsigned int seed, int *hist_size,
                                                int keep_multisets, double **multisets, int64_t *num_tuples,
                                                int offset, int stride)
{
    int flat_len = 0;
    int64_t *flat = legacy_flat(DRESSX_NABLA, g, k, iterations, epsilon, n_samples, seed,
                                hist_size ? &flat_len : nullptr, keep_multisets, multisets, num_tuples, offset,
                                stride);
    return flat_to_pairs(flat, flat_len, hist_size);
}

dress_hist_pair_t *dress_nabla_fit_cuda(p_dress_graph_t g, int k, int iterations, double epsilon, int n_samples,
                                        unsigned int seed, int *hist_size, int keep_multisets,
                                        double **multisets, int64_t *num_tuples)
{
    return dress_nabla_fit_cuda_strided(g, k, iterations, epsilon, n_samples, seed, hist_size, keep_multisets,
                                        multisets, num_tuples, 0, 1);
}

}  // extern "C"

// ---- prepared batches ------------------------------------------------------------------
struct dressx_batch {
    std::vector<dress::Prep> preps;
    std::vector<dress::Prep *> ptrs;
    dress::BatchPlan plan;
    bool ran = false;
};

namespace dress {
namespace {
Status batch_create(dressx_hist_request_t *reqs, int n, dressx_batch_t **out)
{
    Engine &en = engine();
    std::lock_guard<std::mutex> lk(en.mu);
    DRESS_TRY(en.init());
    DRESS_CUDA_TRY(cudaSetDevice(en.device));
    dressx_batch_t *b = new dressx_batch_t();
    b->preps.resize((size_t)n);
    std::vector<Status> pst((size_t)n);
    parallel_for(n, host_threads(n / 8), [&](long long ii) {
        const size_t i = (size_t)ii;
        b->preps[i].r = &reqs[i];
        reqs[i].status = DRESSX_OK;
        reqs[i].hist_flat = nullptr;
        reqs[i].hist_len = 0;
        reqs[i].multisets = nullptr;
        pst[i] = prepare(b->preps[i]);
    }, 8);
    for (int i = 0; i < n; ++i) {
        Prep &p = b->preps[(size_t)i];
        Status s = pst[(size_t)i];
        if (s.ok() && (p.inplace || (!p.empty && !p.batchable)))
            s = Status::Err(DRESSX_EUNSUPPORTED, "request needs the per-subgraph or in-place path");
        if (!s.ok()) {
            for (auto &q : b->preps) std::free(q.ms_host);
            delete b;
            return s;
        }
        if (!p.empty) b->ptrs.push_back(&p);
    }
    if (!b->ptrs.empty()) {
        Status s = plan_batched(b->ptrs, en.ctx, b->plan);
        if (!s.ok()) {
            for (auto &q : b->preps) std::free(q.ms_host);
            delete b;
            return s;
        }
    }
    *out = b;
    return Status::Ok();
}
}  // namespace
}  // namespace dress

extern "C" {

int dressx_batch_create(dressx_hist_request_t *reqs, int n, dressx_batch_t **out)
{
    if (!reqs || n < 0 || !out) return DRESSX_EINVAL;
    *out = nullptr;
    Status s = batch_create(reqs, n, out);
    set_last_error(s);
    return s.code;
}

int dressx_batch_run(dressx_batch_t *b)
{
    if (!b) return DRESSX_EINVAL;
    Engine &en = engine();
    std::lock_guard<std::mutex> lk(en.mu);
    Status s = b->ptrs.empty() ? Status::Ok() : exec_batched(b->plan, en.ctx);
    b->ran = s.ok();
    set_last_error(s);
    return s.code;
}

int dressx_batch_autotune(dressx_batch_t *b, int *group_threads, int *ctas_per_sm, float *rates)
{
    if (!b) return DRESSX_EINVAL;
    Engine &en = engine();
    std::lock_guard<std::mutex> lk(en.mu);
    std::vector<float> r;
    int best = b->ptrs.empty() ? 0 : b->plan.L.gsize;
    Status s = b->ptrs.empty() ? Status::Ok() : autotune_batched(b->plan, en.ctx, &best, &r);
    if (group_threads) *group_threads = best;
    if (ctas_per_sm) *ctas_per_sm = b->plan.tuned_per_sm;
    if (rates)
        for (int i = 0; i < 8; ++i) rates[i] = i < (int)r.size() ? r[(size_t)i] : 0.f;
    set_last_error(s);
    return s.code;
}

int dressx_batch_capture(dressx_batch_t *b)
{
    if (!b) return DRESSX_EINVAL;
    Engine &en = engine();
    std::lock_guard<std::mutex> lk(en.mu);
    Status s = b->ptrs.empty() ? Status::Ok() : capture_batched(b->plan, en.ctx);
    set_last_error(s);
    return s.code;
}

int dressx_batch_fetch(dressx_batch_t *b)
{
    if (!b || !b->ran) return DRESSX_EINVAL;
    Engine &en = engine();
    std::lock_guard<std::mutex> lk(en.mu);
    Status s = b->ptrs.empty() ? Status::Ok() : collect_batched(b->plan, en.ctx);
    for (auto &p : b->preps) {
        if (!s.ok()) break;
        std::free(p.r->hist_flat);
        p.r->hist_flat = nullptr;
        std::free(p.r->multisets);
        p.r->multisets = nullptr;
        double *ms = p.ms_host;
        if (ms) {
            // hand the caller a copy so the batch can be fetched again
            size_t len = (size_t)p.total * (size_t)p.E;
            p.ms_host = (double *)std::malloc((len ? len : 1) * sizeof(double));
            if (p.ms_host) std::memcpy(p.ms_host, ms, len * sizeof(double));
        }
        s = finish(p);
        p.ms_host = ms;
    }
    set_last_error(s);
    return s.code;
}

int dressx_batch_stats(dressx_batch_t *b, int64_t *fits, int64_t *sweeps, int64_t *edge_updates)
{
    if (!b || !b->ran) return DRESSX_EINVAL;
    long long f = 0, sw = 0, eu = 0;
    const size_t n = b->ptrs.size();
    for (size_t i = 0; i < n && b->plan.stats.size() >= 4 * n; ++i) {
        sw += (long long)b->plan.stats[ST_WORDS * (size_t)i + ST_SWEEPS];
        eu += (long long)b->plan.stats[ST_WORDS * (size_t)i + ST_EDGE_ITERS];
        f += (long long)b->plan.stats[ST_WORDS * (size_t)i + ST_FITS];
    }
    if (fits) *fits = f;
    if (sweeps) *sweeps = sw;
    if (edge_updates) *edge_updates = eu;
    return DRESSX_OK;
}

int dressx_batch_timing(dressx_batch_t *b, double *fit_ms, double *hist_ms)
{
    if (!b || !b->ran) return DRESSX_EINVAL;
    if (fit_ms) *fit_ms = b->plan.fit_ms;
    if (hist_ms) *hist_ms = b->plan.hist_ms;
    return DRESSX_OK;
}

void dressx_batch_destroy(dressx_batch_t *b)
{
    if (!b) return;
    Engine &en = engine();
    std::lock_guard<std::mutex> lk(en.mu);
    for (auto &p : b->preps) {
        std::free(p.ms_host);
        std::free(p.hist_mal);
    }
    delete b;
    cudaStreamSynchronize(en.ctx.st);
}

}  // extern "C"
