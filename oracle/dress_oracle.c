/*
 * dress_oracle.c -- CPU restatement of libdress's DRESS hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the B200
 * engine: only the test-suite, the smoke check and the CPU-baseline leg of
 * the benchmark load it.  Nothing in the product library links or calls it.
 *
 * It restates, in plain sequential C, the algorithm of the reference
 * (velicast/dress-graph, libdress/src):
 *   - graph construction              dress.c:103-296, 378-427
 *   - intercept tables                dress.c:307-363
 *   - sorted Kahan-Babuska-Neumaier   dress.c:51-66
 *   - fixed-point fit                 dress.c:452-608
 *   - Delta^k driver                  delta_dress_impl.c:33-318
 *   - Nabla^k driver                  nabla_dress_impl.c:39-311
 *   - exact (value,count) histogram   dress_histogram.c:40-155
 * Every function below names the lines it follows.  It is compiled with
 * -ffp-contract=off so no product is fused into an FMA, exactly like the
 * reference's own -O3 build on baseline x86-64.
 *
 * Parity of this restatement is pinned against (a) the reference library
 * compiled from its own sources into oracle/_ref and (b) the committed
 * golden fixtures in tests/golden, which that library produced.
 */
#include "dress_b200.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ */
/* sorted KBN sum (dress.c:51-66)                                       */
/* ------------------------------------------------------------------ */

static int cmp_double_asc(const void *a, const void *b)
{
    double x = *(const double *)a, y = *(const double *)b;
    return (x > y) - (x < y);
}

/* Ascending sort, then compensated sequential sum.  The branch on the
 * magnitudes picks which operand's low part is recovered (Neumaier). */
double oracle_kbn_sorted_sum(double *terms, int n)
{
    if (n <= 0) return 0.0;
    qsort(terms, (size_t)n, sizeof(double), cmp_double_asc);
    double s = terms[0], c = 0.0;
    for (int i = 1; i < n; ++i) {
        double b = terms[i];
        double t = s + b;
        if (fabs(s) >= fabs(b)) c += (s - t) + b;
        else                    c += (b - t) + s;
        s = t;
    }
    return s + c;
}

/* ------------------------------------------------------------------ */
/* graph construction (dress.c:103-296, 378-427)                        */
/* ------------------------------------------------------------------ */

typedef struct { int x; int e; double w; int seq; } slot_t;

/* Rows are ordered by neighbour id; equal ids keep insertion order (the
 * reference sorts with glibc qsort, a stable merge sort). */
static int cmp_slot(const void *a, const void *b)
{
    const slot_t *p = (const slot_t *)a, *q = (const slot_t *)b;
    if (p->x != q->x) return (p->x > q->x) - (p->x < q->x);
    return (p->seq > q->seq) - (p->seq < q->seq);
}

/* Classic lower/upper bisection over a sorted raw row, as dress.c:70-87. */
static int raw_find(const int *off, const slot_t *raw, int u, int v)
{
    int lo = off[u], hi = off[u + 1] - 1;
    while (lo <= hi) {
        int mid = lo + (hi - lo) / 2;
        int x = raw[mid].x;
        if (x == v) return mid;
        if (x < v) lo = mid + 1; else hi = mid - 1;
    }
    return -1;
}

static void sort_rows(slot_t *s, const int *off, int N)
{
    for (int u = 0; u < N; ++u) {
        int n = off[u + 1] - off[u];
        for (int j = 0; j < n; ++j) s[off[u] + j].seq = j;
        if (n > 1) qsort(s + off[u], (size_t)n, sizeof(slot_t), cmp_slot);
    }
}

p_dress_graph_t oracle_init_graph(int N, int E, int *U, int *V, double *W,
                                  double *NW, dress_variant_t variant,
                                  int precompute_intercepts)
{
    p_dress_graph_t g = (p_dress_graph_t)calloc(1, sizeof(dress_graph_t));
    g->variant = variant; g->N = N; g->E = E; g->U = U; g->V = V; g->W = W;
    g->precompute_intercepts = precompute_intercepts;
    g->vertex_dress = (double *)malloc((size_t)(N > 0 ? N : 1) * sizeof(double));
    if (NW) g->NW = NW;
    else {
        g->NW = (double *)malloc((size_t)(N > 0 ? N : 1) * sizeof(double));
        for (int i = 0; i < N; ++i) g->NW[i] = 1.0;
    }

    /* raw adjacency: both directions for UNDIRECTED, out-edges otherwise */
    int *roff = (int *)calloc((size_t)N + 1, sizeof(int));
    for (int e = 0; e < E; ++e) {
        roff[U[e] + 1]++;
        if (variant == DRESS_VARIANT_UNDIRECTED) roff[V[e] + 1]++;
    }
    for (int i = 0; i < N; ++i) roff[i + 1] += roff[i];
    int Sraw = roff[N];
    slot_t *raw = (slot_t *)malloc((size_t)(Sraw > 0 ? Sraw : 1) * sizeof(slot_t));
    int *fill = (int *)calloc((size_t)N + 1, sizeof(int));
    for (int e = 0; e < E; ++e) {
        double w = W ? W[e] : 1.0;
        int u = U[e], v = V[e];
        slot_t a = { v, e, w, 0 };
        raw[roff[u] + fill[u]++] = a;
        if (variant == DRESS_VARIANT_UNDIRECTED) {
            slot_t b = { u, e, w, 0 };
            raw[roff[v] + fill[v]++] = b;
        }
    }
    sort_rows(raw, roff, N);

    /* variant adjacency: first count, then fill walking raw rows in order */
    int *voff = (int *)calloc((size_t)N + 1, sizeof(int));
    for (int u = 0; u < N; ++u) {
        for (int i = roff[u]; i < roff[u + 1]; ++i) {
            int v = raw[i].x;
            switch (variant) {
            case DRESS_VARIANT_UNDIRECTED: voff[u + 1]++; break;
            case DRESS_VARIANT_FORWARD:    voff[u + 1]++; break;
            case DRESS_VARIANT_BACKWARD:   voff[v + 1]++; break;
            case DRESS_VARIANT_DIRECTED:
                voff[u + 1]++;
                if (raw_find(roff, raw, v, u) < 0) voff[v + 1]++;
                break;
            }
        }
    }
    int maxdeg = 0;
    for (int i = 0; i < N; ++i) {
        if (voff[i + 1] > maxdeg) maxdeg = voff[i + 1];
        voff[i + 1] += voff[i];
    }
    int S = voff[N];
    slot_t *vs = (slot_t *)malloc((size_t)(S > 0 ? S : 1) * sizeof(slot_t));
    memset(fill, 0, ((size_t)N + 1) * sizeof(int));
    for (int u = 0; u < N; ++u) {
        for (int i = roff[u]; i < roff[u + 1]; ++i) {
            int v = raw[i].x, e = raw[i].e;
            double w = raw[i].w;
            if (variant == DRESS_VARIANT_UNDIRECTED) {
                slot_t a = { v, e, 2.0 * w, 0 };
                vs[voff[u] + fill[u]++] = a;
            } else if (variant == DRESS_VARIANT_FORWARD) {
                slot_t a = { v, e, w, 0 };
                vs[voff[u] + fill[u]++] = a;
            } else if (variant == DRESS_VARIANT_BACKWARD) {
                slot_t a = { u, e, w, 0 };
                vs[voff[v] + fill[v]++] = a;
            } else {
                int r = raw_find(roff, raw, v, u);
                slot_t a = { v, e, w, 0 };
                if (r >= 0) a.w = w + raw[r].w;
                vs[voff[u] + fill[u]++] = a;
                if (r < 0) {
                    slot_t b = { u, e, w, 0 };
                    vs[voff[v] + fill[v]++] = b;
                }
            }
        }
    }
    free(raw); free(roff); free(fill);
    sort_rows(vs, voff, N);

    g->adj_offset = voff;
    g->max_degree = maxdeg;
    g->adj_target = (int *)malloc((size_t)(S > 0 ? S : 1) * sizeof(int));
    g->adj_edge_idx = (int *)malloc((size_t)(S > 0 ? S : 1) * sizeof(int));
    g->edge_weight = (double *)malloc((size_t)(E > 0 ? E : 1) * sizeof(double));
    for (int s = 0; s < S; ++s) {
        g->adj_target[s] = vs[s].x;
        g->adj_edge_idx[s] = vs[s].e;
        g->edge_weight[vs[s].e] = vs[s].w;   /* row-major: last slot wins */
    }
    free(vs);

    g->edge_dress = (double *)malloc((size_t)(E > 0 ? E : 1) * sizeof(double));
    g->edge_dress_next = (double *)malloc((size_t)(E > 0 ? E : 1) * sizeof(double));
    for (int e = 0; e < E; ++e) { g->edge_dress[e] = 1.0; g->edge_dress_next[e] = 1.0; }

    if (precompute_intercepts) {
        /* common neighbours by merge walk (dress.c:307-363) */
        int *io = (int *)calloc((size_t)E + 1, sizeof(int));
        for (int pass = 0; pass < 2; ++pass) {
            for (int e = 0; e < E; ++e) {
                int iu = voff[U[e]], iu_end = voff[U[e] + 1];
                int iv = voff[V[e]], iv_end = voff[V[e] + 1];
                int k = pass ? io[e] : 0;
                while (iu < iu_end && iv < iv_end) {
                    int x = g->adj_target[iu], y = g->adj_target[iv];
                    if (x == y) {
                        if (pass) {
                            g->intercept_edge_ux[k] = g->adj_edge_idx[iu];
                            g->intercept_edge_vx[k] = g->adj_edge_idx[iv];
                        }
                        ++k;
                    }
                    iu += (x <= y);
                    iv += (x >= y);
                }
                if (!pass) io[e + 1] = k;
            }
            if (!pass) {
                for (int e = 0; e < E; ++e) io[e + 1] += io[e];
                int T = io[E];
                g->intercept_edge_ux = (int *)malloc((size_t)(T > 0 ? T : 1) * sizeof(int));
                g->intercept_edge_vx = (int *)malloc((size_t)(T > 0 ? T : 1) * sizeof(int));
            }
        }
        g->intercept_offset = io;
    }
    return g;
}

void oracle_free_graph(p_dress_graph_t g)
{
    if (!g) return;
    free(g->adj_offset); free(g->adj_target); free(g->adj_edge_idx);
    free(g->W); free(g->edge_weight); free(g->edge_dress); free(g->edge_dress_next);
    free(g->vertex_dress); free(g->NW);
    if (g->precompute_intercepts) {
        free(g->intercept_offset); free(g->intercept_edge_ux); free(g->intercept_edge_vx);
    }
    free(g->U); free(g->V); free(g);
}

/* ------------------------------------------------------------------ */
/* fit (dress.c:452-608)                                                */
/* ------------------------------------------------------------------ */

/* Numerator terms of edge e: one per common neighbour, then the
 * self-loop / own-edge term (dress.c:452-529). */
static double edge_update(p_dress_graph_t g, int e, double *buf)
{
    int u = g->U[e], v = g->V[e];
    const double *w = g->edge_weight, *d = g->edge_dress;
    int n = 0;
    if (g->precompute_intercepts) {
        for (int k = g->intercept_offset[e]; k < g->intercept_offset[e + 1]; ++k) {
            int a = g->intercept_edge_ux[k], b = g->intercept_edge_vx[k];
            buf[n++] = w[a] * d[a] + w[b] * d[b];
        }
    } else {
        int iu = g->adj_offset[u], iu_end = g->adj_offset[u + 1];
        int iv = g->adj_offset[v], iv_end = g->adj_offset[v + 1];
        while (iu < iu_end && iv < iv_end) {
            int x = g->adj_target[iu], y = g->adj_target[iv];
            if (x == y) {
                int a = g->adj_edge_idx[iu], b = g->adj_edge_idx[iv];
                buf[n++] = w[a] * d[a] + w[b] * d[b];
            }
            iu += (x <= y);
            iv += (x >= y);
        }
    }
    double own = w[e] * d[e];
    if (g->variant == DRESS_VARIANT_FORWARD || g->variant == DRESS_VARIANT_BACKWARD)
        buf[n++] = 4.0 * g->NW[u] + own;
    else
        buf[n++] = 4.0 * g->NW[u] + 4.0 * g->NW[v] + 2.0 * own;
    double num = oracle_kbn_sorted_sum(buf, n);
    double den = g->vertex_dress[u] * g->vertex_dress[v];
    return den > 0.0 ? num / den : 0.0;
}

void oracle_fit(p_dress_graph_t g, int max_iterations, double epsilon,
                int *iterations, double *delta)
{
    int N = g->N, E = g->E;
    double *buf = (double *)malloc(((size_t)g->max_degree + 2) * sizeof(double));
    for (int it = 0; it < max_iterations; ++it) {
        for (int u = 0; u < N; ++u) {                        /* dress.c:556-574 */
            int b = g->adj_offset[u], n = g->adj_offset[u + 1] - b;
            buf[0] = 4.0 * g->NW[u];
            for (int i = 0; i < n; ++i) {
                int ei = g->adj_edge_idx[b + i];
                buf[i + 1] = g->edge_weight[ei] * g->edge_dress[ei];
            }
            g->vertex_dress[u] = sqrt(oracle_kbn_sorted_sum(buf, n + 1));
        }
        double maxd = 0.0;
        for (int e = 0; e < E; ++e) {                        /* dress.c:577-591 */
            double next = edge_update(g, e, buf);
            g->edge_dress_next[e] = next;
            double dd = fabs(g->edge_dress[e] - next);
            if (dd > maxd) maxd = dd;
        }
        double *t = g->edge_dress;                           /* dress.c:594-604 */
        g->edge_dress = g->edge_dress_next;
        g->edge_dress_next = t;
        if (delta) *delta = maxd;
        if (maxd < epsilon) {
            if (iterations) *iterations = it;
            free(buf);
            return;
        }
    }
    if (iterations) *iterations = max_iterations;
    free(buf);
}

/* ------------------------------------------------------------------ */
/* exact histogram (dress_histogram.c:40-155)                           */
/* ------------------------------------------------------------------ */

typedef struct { double *v; size_t n, cap; } valbuf_t;

static void vb_push(valbuf_t *b, double x)
{
    if (b->n == b->cap) {
        b->cap = b->cap ? 2 * b->cap : 1024;
        b->v = (double *)realloc(b->v, b->cap * sizeof(double));
    }
    b->v[b->n++] = x;
}

/* The order-preserving image of a double's bits: ascending by value,
 * -0 before +0, NaNs at the ends by their bits. */
static uint64_t ordered_bits(double x)
{
    uint64_t u;
    memcpy(&u, &x, sizeof u);
    return (u >> 63) ? ~u : (u | 0x8000000000000000ULL);
}

static int cmp_ordered_bits(const void *a, const void *b)
{
    uint64_t x = ordered_bits(*(const double *)a), y = ordered_bits(*(const double *)b);
    return (x > y) - (x < y);
}

/* The flat [bits, count, ...] list of the reference's hash map
 * (dress_histogram.c:40-60, 124-155), ascending by value.  The map keys
 * values by their bits (the hash reads the bit pattern) and merges them by
 * ==, so the only ==-equal values it can keep apart are +0 and -0: they hash
 * to different slots and merge only when one's probe run reaches the other.
 * Here they are two entries, -0 first; a NaN (never == itself) is an entry of
 * its own each time, as in the map. */
static int64_t *vb_flatten(valbuf_t *b, int *hist_size)
{
    if (b->n == 0) { *hist_size = 0; free(b->v); return NULL; }
    qsort(b->v, b->n, sizeof(double), cmp_ordered_bits);
    int64_t *out = (int64_t *)malloc(2 * b->n * sizeof(int64_t));
    size_t m = 0, i = 0;
    while (i < b->n) {
        size_t j = i + 1;
        while (j < b->n && b->v[j] == b->v[i] && ordered_bits(b->v[j]) == ordered_bits(b->v[i])) ++j;
        memcpy(&out[2 * m], &b->v[i], sizeof(double));
        out[2 * m + 1] = (int64_t)(j - i);
        ++m; i = j;
    }
    free(b->v);
    *hist_size = (int)(2 * m);
    return (int64_t *)realloc(out, 2 * m * sizeof(int64_t));
}

/* ------------------------------------------------------------------ */
/* enumeration helpers (delta_dress_impl.h:21-25, delta_dress_impl.c:    */
/* 132-157, nabla_dress_impl.c:111-128)                                 */
/* ------------------------------------------------------------------ */

int64_t oracle_binom(int n, int k)
{
    if (k < 0 || k > n) return 0;
    if (k == 0 || k == n) return 1;
    if (k > n - k) k = n - k;
    int64_t r = 1;
    for (int i = 0; i < k; ++i) r = r * (n - i) / (i + 1);
    return r;
}

int64_t oracle_perm_count(int n, int k)
{
    if (k < 0 || k > n) return 0;
    int64_t r = 1;
    for (int i = 0; i < k; ++i) r *= (n - i);
    return r;
}

static int lcg15(unsigned int *s)
{
    *s = *s * 1103515245u + 12345u;
    return (int)((*s >> 16) & 0x7fff);
}

static int cmp_i64(const void *a, const void *b)
{
    int64_t x = *(const int64_t *)a, y = *(const int64_t *)b;
    return (x > y) - (x < y);
}

/* Sorted, de-duplicated sample indices within this stride; the first LCG
 * draw forms the high 31-bit part (delta_dress_impl.c:234-254). */
int oracle_sample_picks(int64_t per_stride, int n_samples, unsigned int seed,
                        int offset, int64_t **picks_out)
{
    int64_t lim = n_samples < per_stride ? n_samples : per_stride;
    int64_t *p = (int64_t *)malloc((size_t)(lim > 0 ? lim : 1) * sizeof(int64_t));
    unsigned int s = seed + (unsigned int)offset;
    for (int64_t i = 0; i < lim; ++i) {
        int64_t hi = lcg15(&s);
        int64_t lo = lcg15(&s);
        int64_t r = (hi << 31) | lo;
        p[i] = (r & 0x7FFFFFFFFFFFFFFFLL) % per_stride;
    }
    qsort(p, (size_t)lim, sizeof(int64_t), cmp_i64);
    int64_t m = 0;
    for (int64_t i = 0; i < lim; ++i)
        if (i == 0 || p[i] != p[i - 1]) p[m++] = p[i];
    *picks_out = p;
    return (int)m;
}

/* ------------------------------------------------------------------ */
/* Delta^k (delta_dress_impl.c:33-318)                                  */
/* ------------------------------------------------------------------ */

/* Vertex-deleted subgraph: survivors renumbered in order, surviving
 * edges kept in input order, raw W copied, vertex weights reset to 1. */
static p_dress_graph_t delete_vertices(p_dress_graph_t g, const int *del, int k,
                                       int *edge_map)
{
    int N = g->N, E = g->E;
    int *vm = (int *)malloc((size_t)(N > 0 ? N : 1) * sizeof(int));
    for (int v = 0, di = 0, nid = 0; v < N; ++v) {
        if (di < k && v == del[di]) { vm[v] = -1; ++di; }
        else vm[v] = nid++;
    }
    int sE = 0;
    for (int e = 0; e < E; ++e) sE += (vm[g->U[e]] >= 0 && vm[g->V[e]] >= 0);
    if (sE == 0) {
        if (edge_map) for (int e = 0; e < E; ++e) edge_map[e] = -1;
        free(vm);
        return NULL;
    }
    int *sU = (int *)malloc((size_t)sE * sizeof(int));
    int *sV = (int *)malloc((size_t)sE * sizeof(int));
    double *sW = g->W ? (double *)malloc((size_t)sE * sizeof(double)) : NULL;
    for (int e = 0, j = 0; e < E; ++e) {
        int a = vm[g->U[e]], b = vm[g->V[e]];
        if (a >= 0 && b >= 0) {
            sU[j] = a; sV[j] = b;
            if (sW) sW[j] = g->W[e];
            if (edge_map) edge_map[e] = j;
            ++j;
        } else if (edge_map) edge_map[e] = -1;
    }
    free(vm);
    return oracle_init_graph(N - k, sE, sU, sV, sW, NULL, g->variant,
                             g->precompute_intercepts);
}

int64_t *oracle_delta_fit_flat(p_dress_graph_t g, int k, int iterations,
                               double epsilon, int n_samples, unsigned int seed,
                               int *hist_size, int keep_multisets,
                               double **multisets, int64_t *num_subgraphs,
                               int offset, int stride)
{
    int N = g->N, E = g->E, hs = 0;
    valbuf_t vb = { 0, 0, 0 };
    int64_t cnk = k == 0 ? 1 : oracle_binom(N, k);
    if (num_subgraphs) *num_subgraphs = cnk;
    int want_ms = keep_multisets && multisets;
    double *ms = NULL;
    if (want_ms) {
        size_t len = (size_t)cnk * (size_t)E;
        ms = (double *)malloc((len > 0 ? len : 1) * sizeof(double));
        for (size_t i = 0; i < len; ++i) ms[i] = NAN;
        *multisets = ms;
    }
    if (k == 0) {
        if (offset == 0) {
            oracle_fit(g, iterations, epsilon, NULL, NULL);
            for (int e = 0; e < E; ++e) {
                vb_push(&vb, g->edge_dress[e]);
                if (want_ms) ms[e] = g->edge_dress[e];
            }
        }
    } else if (k < N) {
        int64_t per = (cnk + stride - 1 - offset) / stride;
        int64_t *picks = NULL;
        int npicks = 0, pi = 0;
        int sampling = n_samples > 0 && n_samples < per;
        if (sampling) npicks = oracle_sample_picks(per, n_samples, seed, offset, &picks);
        int *combo = (int *)malloc((size_t)k * sizeof(int));
        int *emap = want_ms ? (int *)malloc((size_t)(E > 0 ? E : 1) * sizeof(int)) : NULL;
        /* lexicographic combinations; s = rank, my_s = rank within stride */
        for (int i = 0; i < k; ++i) combo[i] = i;
        int64_t s = 0, my_s = 0;
        for (;;) {
            if (s % stride == offset) {
                int go = !sampling || (pi < npicks && my_s == picks[pi]);
                if (sampling && go) ++pi;
                if (go) {
                    p_dress_graph_t sub = delete_vertices(g, combo, k, emap);
                    if (sub) {
                        oracle_fit(sub, iterations, epsilon, NULL, NULL);
                        for (int e = 0; e < sub->E; ++e) vb_push(&vb, sub->edge_dress[e]);
                        if (want_ms)
                            for (int e = 0; e < E; ++e)
                                ms[(size_t)s * E + e] = emap[e] >= 0 ? sub->edge_dress[emap[e]] : NAN;
                        oracle_free_graph(sub);
                    }
                }
                ++my_s;
                if (sampling && pi >= npicks) break;
            }
            ++s;
            int i = k - 1;
            while (i >= 0 && combo[i] == N - k + i) --i;
            if (i < 0) break;
            ++combo[i];
            for (int j = i + 1; j < k; ++j) combo[j] = combo[j - 1] + 1;
        }
        free(combo); free(emap); free(picks);
    }
    if (!hist_size) { free(vb.v); return NULL; }
    int64_t *flat = vb_flatten(&vb, &hs);
    *hist_size = hs;
    return flat;
}

/* ------------------------------------------------------------------ */
/* Nabla^k (nabla_dress_impl.c:39-311)                                  */
/* ------------------------------------------------------------------ */

/* Marker weight of tuple position i: sqrt of the (i+1)-th prime for the
 * first sixteen positions, sqrt(2i+3) beyond (nabla_dress_impl.c:33-46). */
double oracle_marker_weight(int i)
{
    static const int pr[16] = { 2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53 };
    return i < 16 ? sqrt((double)pr[i]) : sqrt((double)(2 * i + 3));
}

int64_t *oracle_nabla_fit_flat(p_dress_graph_t g, int k, int iterations,
                               double epsilon, int n_samples, unsigned int seed,
                               int *hist_size, int keep_multisets,
                               double **multisets, int64_t *num_tuples,
                               int offset, int stride)
{
    int N = g->N, E = g->E, hs = 0;
    valbuf_t vb = { 0, 0, 0 };
    int64_t pnk = k == 0 ? 1 : oracle_perm_count(N, k);
    if (num_tuples) *num_tuples = pnk;
    int want_ms = keep_multisets && multisets;
    double *ms = NULL;
    if (want_ms) {
        size_t len = (size_t)pnk * (size_t)E;
        ms = (double *)malloc((len > 0 ? len : 1) * sizeof(double));
        for (size_t i = 0; i < len; ++i) ms[i] = NAN;
        *multisets = ms;
    }
    if (k == 0) {
        if (offset == 0) {
            oracle_fit(g, iterations, epsilon, NULL, NULL);
            for (int e = 0; e < E; ++e) {
                vb_push(&vb, g->edge_dress[e]);
                if (want_ms) ms[e] = g->edge_dress[e];
            }
        }
    } else if (k < N) {
        int64_t per = (pnk + stride - 1 - offset) / stride;
        int64_t *picks = NULL;
        int npicks = 0, pi = 0;
        int sampling = n_samples > 0 && n_samples < per;
        if (sampling) npicks = oracle_sample_picks(per, n_samples, seed, offset, &picks);
        int *tup = (int *)malloc((size_t)k * sizeof(int));
        char *used = (char *)calloc((size_t)N, 1);
        /* lexicographic ordered tuples without repetition */
        for (int i = 0; i < k; ++i) { tup[i] = i; used[i] = 1; }
        int64_t s = 0, my_s = 0;
        for (;;) {
            if (s % stride == offset) {
                int go = !sampling || (pi < npicks && my_s == picks[pi]);
                if (sampling && go) ++pi;
                if (go) {
                    int *mU = (int *)malloc((size_t)(E > 0 ? E : 1) * sizeof(int));
                    int *mV = (int *)malloc((size_t)(E > 0 ? E : 1) * sizeof(int));
                    memcpy(mU, g->U, (size_t)E * sizeof(int));
                    memcpy(mV, g->V, (size_t)E * sizeof(int));
                    double *mW = NULL;
                    if (g->W) {
                        mW = (double *)malloc((size_t)(E > 0 ? E : 1) * sizeof(double));
                        memcpy(mW, g->W, (size_t)E * sizeof(double));
                    }
                    double *mNW = (double *)malloc((size_t)N * sizeof(double));
                    for (int v = 0; v < N; ++v) mNW[v] = 1.0;
                    for (int i = 0; i < k; ++i) mNW[tup[i]] = oracle_marker_weight(i);
                    p_dress_graph_t m = oracle_init_graph(N, E, mU, mV, mW, mNW,
                                                          g->variant, g->precompute_intercepts);
                    oracle_fit(m, iterations, epsilon, NULL, NULL);
                    for (int e = 0; e < E; ++e) {
                        vb_push(&vb, m->edge_dress[e]);
                        if (want_ms) ms[(size_t)s * E + e] = m->edge_dress[e];
                    }
                    oracle_free_graph(m);
                }
                ++my_s;
                if (sampling && pi >= npicks) break;
            }
            ++s;
            /* advance to the next tuple: bump the deepest position that can
             * take a larger unused vertex, then refill the tail minimally */
            int i = k - 1, ok = 0;
            while (i >= 0) {
                used[tup[i]] = 0;
                int c = tup[i] + 1;
                while (c < N && used[c]) ++c;
                if (c < N) { tup[i] = c; used[c] = 1; ok = 1; break; }
                --i;
            }
            if (!ok) break;
            for (int j = i + 1; j < k; ++j) {
                int c = 0;
                while (used[c]) ++c;
                tup[j] = c; used[c] = 1;
            }
        }
        free(tup); free(used); free(picks);
    }
    if (!hist_size) { free(vb.v); return NULL; }
    int64_t *flat = vb_flatten(&vb, &hs);
    *hist_size = hs;
    return flat;
}

/* Frees memory that this library returned (histograms, multisets). */
/* ------------------------------------------------------------------ */
/* virtual-edge query (dress.c:651-739)                                  */
/* ------------------------------------------------------------------ */

/* An existing edge returns its value; otherwise the common-neighbour terms of
 * the frozen state plus the self-loop constant are summed (sorted KBN) and
 * the pair's own value is iterated with everything else held fixed. */
double oracle_get(p_dress_graph_t g, int u, int v, int max_iterations, double epsilon, double edge_weight)
{
    int lo = g->adj_offset[u], hi = g->adj_offset[u + 1] - 1;
    while (lo <= hi) {
        int mid = lo + (hi - lo) / 2;
        int nb = g->adj_target[mid];
        if (nb == v) return g->edge_dress[g->adj_edge_idx[mid]];
        if (nb < v) lo = mid + 1;
        else hi = mid - 1;
    }
    int du = g->adj_offset[u + 1] - g->adj_offset[u];
    int dv = g->adj_offset[v + 1] - g->adj_offset[v];
    double *t = (double *)malloc(((du < dv ? du : dv) + 1) * sizeof(double));
    int n = 0;
    int iu = g->adj_offset[u], iu_end = g->adj_offset[u + 1];
    int iv = g->adj_offset[v], iv_end = g->adj_offset[v + 1];
    while (iu < iu_end && iv < iv_end) {
        int x = g->adj_target[iu], y = g->adj_target[iv];
        if (x == y) {
            int eu = g->adj_edge_idx[iu], ev = g->adj_edge_idx[iv];
            t[n++] = g->edge_weight[eu] * g->edge_dress[eu] + g->edge_weight[ev] * g->edge_dress[ev];
        }
        iu += (x <= y);
        iv += (x >= y);
    }
    int fwd = g->variant == DRESS_VARIANT_FORWARD || g->variant == DRESS_VARIANT_BACKWARD;
    double nwu = g->NW ? g->NW[u] : 1.0, nwv = g->NW ? g->NW[v] : 1.0;
    t[n++] = fwd ? 4.0 * nwu : 4.0 * nwu + 4.0 * nwv;
    double A = oracle_kbn_sorted_sum(t, n);
    free(t);
    double cf = fwd ? 1.0 : 2.0;
    double cw = g->variant == DRESS_VARIANT_UNDIRECTED ? 2.0 * edge_weight : edge_weight;
    double du2 = g->vertex_dress[u] * g->vertex_dress[u];
    double dv2 = g->vertex_dress[v] * g->vertex_dress[v];
    if (du2 <= 0.0 || dv2 <= 0.0) return 0.0;
    double d = 1.0;
    for (int it = 0; it < max_iterations; ++it) {
        double wd = cw * d;
        double den = sqrt(du2 + wd) * sqrt(dv2 + wd);
        if (den <= 0.0) return 0.0;
        double nx = (A + cf * wd) / den;
        if (fabs(nx - d) <= epsilon) {
            d = nx;
            break;
        }
        d = nx;
    }
    return d;
}

void oracle_free(void *p) { free(p); }
