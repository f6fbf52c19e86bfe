// graph_host.cpp -- dress_init_graph / dress_free_graph.
//
// Host-side graph construction with the reference's contract
// (libdress/include/dress/dress.h:77-93) and bit-identical output
// (libdress/src/dress.c:103-427): the variant CSR with rows ascending by
// neighbour id (ties keep insertion order, as the reference's stable qsort
// does), the variant weights w-bar, the optional common-neighbour tables, and
// every edge value set to 1.0.  The reference's Python ctypes loader binds
// these two names from the CUDA library (python/src/dress/cuda/__init__.py:143-203),
// so they live here.  Rows are ordered with two stable counting passes
// (by neighbour, then by row) instead of one qsort per row.
#include <cstdlib>
#include <cstring>
#include <vector>

#include "dress_b200.h"

namespace {

struct Slot {
    int row, x, e;
    double w;
};

// Stable counting sort of slots by (row, x): by x first, then by row.
void sort_slots(std::vector<Slot> &s, int N)
{
    std::vector<Slot> tmp(s.size());
    std::vector<long long> cnt((size_t)N + 1);
    for (int pass = 0; pass < 2; ++pass) {
        std::fill(cnt.begin(), cnt.end(), 0);
        for (const Slot &q : s) cnt[(size_t)(pass ? q.row : q.x) + 1]++;
        for (int i = 0; i < N; ++i) cnt[(size_t)i + 1] += cnt[i];
        for (const Slot &q : s) tmp[(size_t)cnt[pass ? q.row : q.x]++] = q;
        s.swap(tmp);
    }
}

// Bisection for neighbour v in row u of the sorted raw adjacency
// (same probe sequence as libdress/src/dress.c:70-87).
long long find_raw(const std::vector<long long> &off, const std::vector<Slot> &raw, int u, int v)
{
    long long lo = off[u], hi = off[(size_t)u + 1] - 1;
    while (lo <= hi) {
        long long mid = lo + (hi - lo) / 2;
        int x = raw[(size_t)mid].x;
        if (x == v) return mid;
        if (x < v) lo = mid + 1;
        else hi = mid - 1;
    }
    return -1;
}

template <class T> T *xmalloc(size_t n) { return (T *)std::malloc((n ? n : 1) * sizeof(T)); }

}  // namespace

extern "C" {

p_dress_graph_t dress_init_graph(int N, int E, int *U, int *V, double *W, double *NW,
                                 dress_variant_t variant, int precompute_intercepts)
{
    if (N < 0 || E < 0 || (E > 0 && (!U || !V))) return nullptr;
    for (int e = 0; e < E; ++e)
        if (U[e] < 0 || U[e] >= N || V[e] < 0 || V[e] >= N) return nullptr;

    p_dress_graph_t g = (p_dress_graph_t)std::calloc(1, sizeof(dress_graph_t));
    g->variant = variant;
    g->N = N;
    g->E = E;
    g->U = U;
    g->V = V;
    g->W = W;
    g->precompute_intercepts = precompute_intercepts;
    g->vertex_dress = xmalloc<double>((size_t)N);
    if (NW) {
        g->NW = NW;
    } else {
        g->NW = xmalloc<double>((size_t)N);
        for (int i = 0; i < N; ++i) g->NW[i] = 1.0;
    }
    const bool und = variant == DRESS_VARIANT_UNDIRECTED;

    // raw adjacency: u->v for every edge, plus v->u when undirected
    std::vector<Slot> raw;
    raw.reserve((size_t)E * (und ? 2 : 1));
    for (int e = 0; e < E; ++e) {
        double w = W ? W[e] : 1.0;
        raw.push_back({U[e], V[e], e, w});
        if (und) raw.push_back({V[e], U[e], e, w});
    }
    sort_slots(raw, N);
    std::vector<long long> roff((size_t)N + 1, 0);
    for (const Slot &q : raw) roff[(size_t)q.row + 1]++;
    for (int i = 0; i < N; ++i) roff[(size_t)i + 1] += roff[i];

    // variant adjacency, generated walking the raw rows in order
    std::vector<Slot> vs;
    vs.reserve(raw.size() * (variant == DRESS_VARIANT_DIRECTED ? 2 : 1));
    for (const Slot &q : raw) {
        int u = q.row, v = q.x;
        switch (variant) {
        case DRESS_VARIANT_UNDIRECTED: vs.push_back({u, v, q.e, 2.0 * q.w}); break;
        case DRESS_VARIANT_FORWARD:    vs.push_back({u, v, q.e, q.w}); break;
        case DRESS_VARIANT_BACKWARD:   vs.push_back({v, u, q.e, q.w}); break;
        case DRESS_VARIANT_DIRECTED: {
            long long r = find_raw(roff, raw, v, u);
            vs.push_back({u, v, q.e, r >= 0 ? q.w + raw[(size_t)r].w : q.w});
            if (r < 0) vs.push_back({v, u, q.e, q.w});
            break;
        }
        }
    }
    raw.clear();
    raw.shrink_to_fit();
    sort_slots(vs, N);

    const size_t S = vs.size();
    g->adj_offset = xmalloc<int>((size_t)N + 1);
    g->adj_target = xmalloc<int>(S);
    g->adj_edge_idx = xmalloc<int>(S);
    g->edge_weight = xmalloc<double>((size_t)E);
    std::vector<int> deg((size_t)N, 0);
    for (const Slot &q : vs) deg[(size_t)q.row]++;
    g->adj_offset[0] = 0;
    int maxdeg = 0;
    for (int i = 0; i < N; ++i) {
        g->adj_offset[i + 1] = g->adj_offset[i] + deg[(size_t)i];
        if (deg[(size_t)i] > maxdeg) maxdeg = deg[(size_t)i];
    }
    g->max_degree = maxdeg;
    for (size_t s = 0; s < S; ++s) {
        g->adj_target[s] = vs[s].x;
        g->adj_edge_idx[s] = vs[s].e;
        g->edge_weight[vs[s].e] = vs[s].w;      // row-major: the last slot of an edge wins
    }

    g->edge_dress = xmalloc<double>((size_t)E);
    g->edge_dress_next = xmalloc<double>((size_t)E);
    for (int e = 0; e < E; ++e) g->edge_dress[e] = g->edge_dress_next[e] = 1.0;

    if (precompute_intercepts) {
        // common neighbours by the merge walk of libdress/src/dress.c:307-363
        const int *off = g->adj_offset, *tg = g->adj_target, *ei = g->adj_edge_idx;
        g->intercept_offset = xmalloc<int>((size_t)E + 1);
        std::vector<int> ux, vx;
        g->intercept_offset[0] = 0;
        for (int e = 0; e < E; ++e) {
            int iu = off[U[e]], iu_end = off[U[e] + 1];
            int iv = off[V[e]], iv_end = off[V[e] + 1];
            while (iu < iu_end && iv < iv_end) {
                int x = tg[iu], y = tg[iv];
                if (x == y) { ux.push_back(ei[iu]); vx.push_back(ei[iv]); }
                iu += (x <= y);
                iv += (x >= y);
            }
            g->intercept_offset[e + 1] = (int)ux.size();
        }
        g->intercept_edge_ux = xmalloc<int>(ux.size());
        g->intercept_edge_vx = xmalloc<int>(vx.size());
        if (!ux.empty()) {
            std::memcpy(g->intercept_edge_ux, ux.data(), ux.size() * sizeof(int));
            std::memcpy(g->intercept_edge_vx, vx.data(), vx.size() * sizeof(int));
        }
    }
    return g;
}

void dress_free_graph(p_dress_graph_t g)
{
    if (!g) return;
    std::free(g->adj_offset);
    std::free(g->adj_target);
    std::free(g->adj_edge_idx);
    std::free(g->W);
    std::free(g->edge_weight);
    std::free(g->edge_dress);
    std::free(g->edge_dress_next);
    std::free(g->vertex_dress);
    std::free(g->NW);
    if (g->precompute_intercepts) {
        std::free(g->intercept_offset);
        std::free(g->intercept_edge_ux);
        std::free(g->intercept_edge_vx);
    }
    std::free(g->U);
    std::free(g->V);
    std::free(g);
}

}  // extern "C"
