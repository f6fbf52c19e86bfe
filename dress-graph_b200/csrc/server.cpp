// server.cpp -- a continuous-batching request server over the engine.
//
// The reference has no serving layer: every binding calls dress_fit_cuda or
// the Delta/Nabla drivers once per request, each call uploading its graph,
// fitting on the legacy stream and downloading
// (libdress/src/cuda/dress_cuda.cu:445-707, delta_dress_cuda.c:24-85).
// Here one server object keeps requests of many sizes in flight at once:
//
//   submit (caller's thread)  validate, plan the path and the device bytes,
//                             pack small graphs into the batch kernel's image
//   scheduler thread          admit in arrival order against the memory budget,
//                             upload admitted small requests into the arena,
//                             cut their work into slices and pack slices of
//                             all waiting requests into short persistent batch
//                             launches (a few in flight, on high-priority
//                             streams); a host callback reports each launch's
//                             end, and a request whose last slice has run goes
//                             to a finisher
//   lane threads              large requests (rows above 31 neighbours, state
//                             beyond shared memory): the single-graph fit or
//                             the per-subgraph Delta/Nabla path, each lane on
//                             its own streams, concurrently with the batches
//   finisher threads          histograms and downloads of finished batch
//                             requests, then the completion record
//
// All device memory of served requests comes from one memory pool owned by
// the server (the arena), whose release threshold keeps it resident between
// requests.  A request's numbers do not depend on what it shares the device
// with: every fit is independent and every sum has a fixed order.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "batch.h"
#include "engine.h"
#include "hist.h"

namespace dress {
namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b)
{
    return std::chrono::duration<double, std::milli>(b - a).count();
}

int next_pow2i(int x)
{
    int m = 1;
    while (m < x) m <<= 1;
    return m;
}

// Opt-in shared memory per block of a B200 (used when no device is asked).
constexpr long long B200_SMEM_OPTIN = 232448;
// Device bytes per value of a histogram: the values, the sort's second
// buffer, and the sort / run-length scratch.
constexpr long long HIST_BYTES_PER_VALUE = 56;

// Pinned staging per lane and finisher at start-up (each grows on demand).
constexpr size_t STAGE_START_BYTES = (size_t)64 << 20;

// Largest whole-graph fit packed into batch launches.
constexpr int PLAIN_BATCH_MAX_EDGES = 2048;

// Threads per fit by edge count.
int gsize_for(int E) { return E <= 640 ? 32 : E <= 2048 ? 64 : E <= 8192 ? 128 : 256; }

int class_of(int kind, int path)
{
    const bool fit = kind == DRESSX_FIT;
    if (path == DRESSX_PATH_BATCH) return fit ? DRESSX_CLASS_FIT_BATCH : DRESSX_CLASS_HIST_BATCH;
    return fit ? DRESSX_CLASS_FIT_LANE : DRESSX_CLASS_HIST_LANE;
}

// ---- planning ---------------------------------------------------------------------
struct Planned {
    int path = DRESSX_PATH_NONE;
    long long bytes = 0;                // device bytes reserved at admission
    int item_kind = ITEM_PLAIN;
    long long items = 0;                // fits to run on the batch path
    long long num_subgraphs = 0;
    int N = 0, E = 0, S = 0, T = 0, M = 2, gsize = 32, k = 0;
    int has_nw = 0, has_dinit = 0, fwd = 0;
    ParentLayout PL{};
    std::vector<unsigned char> packed;  // batch path: the parent image
};

Status check_graph(p_dress_graph_t g)
{
    if (!g) return Status::Err(DRESSX_EINVAL, "request without graph");
    if (g->N < 0 || g->E < 0) return Status::Err(DRESSX_EINVAL, "negative graph size");
    if (g->N > 0 && (!g->adj_offset || !g->vertex_dress))
        return Status::Err(DRESSX_EINVAL, "graph without CSR rows");
    if (g->E > 0 && (!g->U || !g->V || !g->edge_weight || !g->edge_dress || !g->adj_target || !g->adj_edge_idx))
        return Status::Err(DRESSX_EINVAL, "graph without edge arrays");
    if (g->N > 0 && (g->adj_offset[0] != 0 || g->adj_offset[g->N] < 0))
        return Status::Err(DRESSX_EINVAL, "bad CSR offsets");
    return Status::Ok();
}

// Conservative device footprint of the single-graph fit (its buffers, the
// common-neighbour pairs bounded by sum_e min(deg u, deg v), the hub scratch).
long long lane_fit_bytes(p_dress_graph_t g, int maxdeg)
{
    const long long N = g->N, E = g->E, S = N > 0 ? g->adj_offset[N] : 0;
    long long T = 0;
    for (long long e = 0; e < E; ++e) {
        const int u = g->U[e], v = g->V[e];
        const long long du = g->adj_offset[u + 1] - g->adj_offset[u];
        const long long dv = g->adj_offset[v + 1] - g->adj_offset[v];
        T += du < dv ? du : dv;
    }
    return 96 * N + 32 * S + 144 * E + 16 * T + 16LL * 148 * maxdeg + (32LL << 20);
}

Status plan_request(p_dress_graph_t g, int kind, int k, long long smem_cap, bool pack, Planned &pl)
{
    DRESS_TRY(check_graph(g));
    if (kind != DRESSX_FIT && kind != DRESSX_DELTA && kind != DRESSX_NABLA)
        return Status::Err(DRESSX_EINVAL, "bad request kind");
    if (kind != DRESSX_FIT && k < 0) return Status::Err(DRESSX_EINVAL, "negative k");
    const int N = g->N, E = g->E, S = N > 0 ? g->adj_offset[N] : 0;
    pl.N = N;
    pl.E = E;
    pl.S = S;
    pl.k = kind == DRESSX_FIT ? 0 : k;
    for (int e = 0; e < E; ++e)
        if (g->U[e] < 0 || g->U[e] >= N || g->V[e] < 0 || g->V[e] >= N)
            return Status::Err(DRESSX_EINVAL, "edge endpoint out of range");
    int maxdeg = 0;
    for (int u = 0; u < N; ++u) maxdeg = std::max(maxdeg, g->adj_offset[u + 1] - g->adj_offset[u]);
    pl.num_subgraphs = kind == DRESSX_FIT ? 0
                     : k == 0 ? 1 : kind == DRESSX_DELTA ? binom_h(N, k) : perm_h(N, k);

    // batch path: one fit's state in shared memory; Delta/Nabla with
    // 1 <= k < N (the other orders are trivial or in-place fits, served by
    // the lane path).  A whole-graph fit keeps rows of at most 256
    // neighbours: one thread sums a row there.
    bool batch = batch_group_bytes(E, N, pl.k, gsize_for(E)) <= smem_cap - 1024 &&
                 batch_group_bytes(E, N, pl.k, gsize_for(E)) <= BATCH_GROUP_BYTES_MAX;
    if (kind == DRESSX_FIT) batch = batch && maxdeg <= 256;
    if (kind != DRESSX_FIT) batch = batch && k >= 1 && k < N;
    // a whole-graph fit in the batch kernel runs on one thread group (one
    // SM); above a few thousand edges the single-graph fit, which spreads
    // every sweep over the whole device, answers sooner
    if (kind == DRESSX_FIT) batch = batch && E <= PLAIN_BATCH_MAX_EDGES;
    std::vector<int> ioff, pairs;
    if (batch) {
        bool dup = false;
        merge_walk_pairs(g, ioff, pairs, maxdeg, dup);
        // masks reproduce the rebuilt subgraph except for the reciprocal-weight
        // lookup of DIRECTED graphs with repeated directed edges
        if (kind != DRESSX_FIT && dup && g->variant == DRESS_VARIANT_DIRECTED) batch = false;
    }
    if (!batch) {
        pl.path = DRESSX_PATH_LANE;
        long long fitb = lane_fit_bytes(g, maxdeg);
        if (kind == DRESSX_FIT) {
            pl.bytes = fitb;
        } else {
            long long subs = k == 0 ? 1 : (k >= N ? 0 : pl.num_subgraphs);
            long long values = subs * (long long)E;
            pl.bytes = fitb + values * HIST_BYTES_PER_VALUE;
        }
        return Status::Ok();
    }

    pl.path = DRESSX_PATH_BATCH;
    pl.T = (int)(pairs.size() / 2);
    pl.M = std::max(2, next_pow2i(maxdeg + 1));
    pl.gsize = gsize_for(E);
    pl.fwd = g->variant == DRESS_VARIANT_FORWARD || g->variant == DRESS_VARIANT_BACKWARD;
    if (kind == DRESSX_FIT) {
        pl.item_kind = ITEM_PLAIN;
        pl.items = 1;
        pl.has_nw = g->NW != nullptr;
        pl.has_dinit = 1;       // a fit continues from the current edge values
    } else {
        pl.item_kind = kind == DRESSX_DELTA ? ITEM_DELTA : ITEM_NABLA;
        pl.items = pl.num_subgraphs;
    }
    pl.PL = parent_layout(N, E, S, pl.T, pl.has_nw, pl.has_dinit);
    const long long out = kind == DRESSX_FIT ? 8LL * (E + N) : 8LL * pl.items * E;
    pl.bytes = pl.PL.bytes + out + 8LL * ST_WORDS + 4096 +
               (kind == DRESSX_FIT ? 0 : pl.items * (long long)E * (HIST_BYTES_PER_VALUE - 8));
    if (!pack) return Status::Ok();
    pl.packed.assign((size_t)pl.PL.bytes, 0);
    unsigned char *b = pl.packed.data();
    if (E) {
        std::memcpy(b + pl.PL.U, g->U, (size_t)E * 4);
        std::memcpy(b + pl.PL.V, g->V, (size_t)E * 4);
        std::memcpy(b + pl.PL.w, g->edge_weight, (size_t)E * 8);
    }
    std::memcpy(b + pl.PL.row_off, g->adj_offset, (size_t)(N + 1) * 4);
    if (S) std::memcpy(b + pl.PL.row_eid, g->adj_edge_idx, (size_t)S * 4);
    std::memcpy(b + pl.PL.ioff, ioff.data(), (size_t)(E + 1) * 4);
    if (pl.T) std::memcpy(b + pl.PL.pairs, pairs.data(), (size_t)pl.T * 8);
    if (pl.has_nw) std::memcpy(b + pl.PL.nw, g->NW, (size_t)N * 8);
    if (pl.has_dinit && E) std::memcpy(b + pl.PL.dinit, g->edge_dress, (size_t)E * 8);
    return Status::Ok();
}

// ---- server state ---------------------------------------------------------------
struct Server;

struct Req {
    dressx_server_request_t *pub = nullptr;
    Planned pl;
    int cls = 0;
    long long seq = 0;
    Clock::time_point t_submit, t_admit;
    bool admitted = false, started = false, cancelled = false, queued_fin = false;
    bool placed = false;        // batch path: uploaded and handed to the scheduler's lists
    long long next_item = 0, items_done = 0;
    int inflight = 0;
    Status err;
    // batch path: resident state in the arena
    DevBuf<unsigned char> d_data;
    DevBuf<unsigned long long> d_values, d_stats;
    ParentDesc desc{};
};

struct Slot {
    Server *srv = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    Pinned host;
    DevBuf<unsigned char> dev;
    std::vector<std::pair<Req *, long long>> credits;
    bool busy = false, finished = false;
    Status err;
};

struct Lane {
    Ctx ctx;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

struct Server {
    dressx_server_config_t cfg{};
    int device = 0, sms = 148;
    long long smem_cap = B200_SMEM_OPTIN - 256;
    long long budget = 0;
    cudaMemPool_t pool = nullptr;
    cudaStream_t up = nullptr;            // uploads of admitted batch requests
    cudaEvent_t up_ev = nullptr, epoch = nullptr;
    std::vector<Slot *> slots;
    std::vector<Lane *> lanes;
    std::vector<Ctx *> fins;
    std::vector<std::thread> threads;

    std::mutex mu;
    std::condition_variable cv_sched, cv_lane, cv_fin, cv_done;
    bool wake = false, stop = false, closing = false;
    std::deque<Req *> waiting, lane_q, fin_q;
    std::vector<Req *> active;            // admitted batch requests with slices to launch
    std::unordered_map<dressx_server_request_t *, Req *> live;
    long long seq = 0;
    long long reserved = 0, peak_reserved = 0;
    int in_service = 0, max_in_service = 0;

    // statistics
    Clock::time_point t0;
    long long submitted = 0, completed = 0, failed = 0, cancelled = 0, rejected = 0;
    long long fits = 0, edge_sweeps = 0, launches = 0;
    std::vector<double> lat[DRESSX_CLASSES], que[DRESSX_CLASSES];
    long long cls_failed[DRESSX_CLASSES] = {0, 0, 0, 0};
    std::vector<std::pair<double, double>> intervals;   // device [start, end) ms after epoch

    Status start(const dressx_server_config_t *c);
    void shutdown();
    void scheduler();
    void lane_main(Lane *ln);
    void fin_main(Ctx *ctx);
    // helpers (mu held unless noted)
    void complete_locked(Req *r, int status);
    bool form_launch(Slot *s, BatchLaunch &L, std::vector<ParentDesc> &descs, std::vector<Chunk> &chunks);
    void credit_locked(Slot *s);
    Status admit_batch(Req *r);                       // mu not held
    Status issue_launch(Slot *s, BatchLaunch &L, const std::vector<ParentDesc> &descs,
                        const std::vector<Chunk> &chunks);   // mu not held
    void record_interval(cudaEvent_t a, cudaEvent_t b);      // mu not held
    void finish_batch(Req *r, Ctx *ctx);              // mu not held
};

void CUDART_CB slot_done(void *arg)
{
    Slot *s = (Slot *)arg;
    Server *sv = s->srv;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        s->finished = true;
        sv->wake = true;
    }
    sv->cv_sched.notify_one();
}

Status Server::start(const dressx_server_config_t *c)
{
    if (c) cfg = *c;
    else cfg.device = -1;
    if (cfg.lanes <= 0) cfg.lanes = 4;
    if (cfg.launch_slots <= 0) cfg.launch_slots = 3;
    if (cfg.launch_work <= 0) cfg.launch_work = 1LL << 21;
    if (cfg.finishers <= 0) cfg.finishers = 2;
    if (cfg.max_queued <= 0) cfg.max_queued = 65536;
    Engine &en = engine();
    {
        std::lock_guard<std::mutex> lk(en.mu);
        DRESS_TRY(en.init());
    }
    device = cfg.device >= 0 ? cfg.device : en.device;
    DRESS_CUDA_TRY(cudaSetDevice(device));
    DRESS_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    int optin = 0;
    DRESS_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
    smem_cap = optin - 256;
    size_t free_b = 0, total_b = 0;
    DRESS_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
    budget = cfg.memory_budget_bytes ? (long long)cfg.memory_budget_bytes
                                     : std::min<long long>(120LL << 30, (long long)(0.9 * (double)free_b));

    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    DRESS_CUDA_TRY(cudaMemPoolCreate(&pool, &props));
    unsigned long long keep = (unsigned long long)budget;
    DRESS_CUDA_TRY(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));

    int lo = 0, hi = 0;     // hi = numerically lowest = most urgent
    DRESS_CUDA_TRY(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    DRESS_CUDA_TRY(cudaStreamCreateWithPriority(&up, cudaStreamNonBlocking, hi));
    DRESS_CUDA_TRY(cudaEventCreateWithFlags(&up_ev, cudaEventDisableTiming));
    DRESS_CUDA_TRY(cudaEventCreate(&epoch));
    DRESS_CUDA_TRY(cudaEventRecord(epoch, up));
    DRESS_CUDA_TRY(cudaEventRecord(up_ev, up));
    DRESS_CUDA_TRY(cudaStreamSynchronize(up));
    for (int i = 0; i < cfg.launch_slots; ++i) {
        Slot *s = new Slot;
        slots.push_back(s);
        s->srv = this;
        DRESS_CUDA_TRY(cudaStreamCreateWithPriority(&s->st, cudaStreamNonBlocking, hi));
        DRESS_CUDA_TRY(cudaEventCreate(&s->ev0));
        DRESS_CUDA_TRY(cudaEventCreate(&s->ev1));
    }
    for (int i = 0; i < cfg.lanes; ++i) {
        Lane *ln = new Lane;
        lanes.push_back(ln);
        DRESS_TRY(ln->ctx.create(device, sms, &en.cfg, lo));
        DRESS_CUDA_TRY(cudaEventCreate(&ln->ev0));
        DRESS_CUDA_TRY(cudaEventCreate(&ln->ev1));
    }
    for (int i = 0; i < cfg.finishers; ++i) {
        Ctx *c2 = new Ctx;
        fins.push_back(c2);
        DRESS_TRY(c2->create(device, sms, &en.cfg, hi));
    }
    // staging buffers pinned now rather than while requests are in flight
    for (Lane *ln : lanes) {
        ln->ctx.stage->reserve(STAGE_START_BYTES);
        ln->ctx.stage2->reserve(2 * STAGE_CHUNK);    // the second upload of a large fit
    }
    for (Ctx *c2 : fins) c2->stage->reserve(STAGE_START_BYTES);
    t0 = Clock::now();
    threads.emplace_back([this] { scheduler(); });
    for (Lane *ln : lanes) threads.emplace_back([this, ln] { lane_main(ln); });
    for (Ctx *c2 : fins) threads.emplace_back([this, c2] { fin_main(c2); });
    return Status::Ok();
}

void Server::shutdown()
{
    {
        std::unique_lock<std::mutex> lk(mu);
        closing = true;
        while (!waiting.empty()) {
            Req *r = waiting.front();
            waiting.pop_front();
            complete_locked(r, DRESSX_ECANCELLED);
        }
        cv_done.wait(lk, [&] { return live.empty(); });
        stop = true;
        wake = true;
    }
    cv_sched.notify_all();
    cv_lane.notify_all();
    cv_fin.notify_all();
    for (auto &t : threads)
        if (t.joinable()) t.join();
    threads.clear();
    cudaSetDevice(device);
    for (Slot *s : slots) {
        if (s->st) cudaStreamSynchronize(s->st);
        s->dev.release();
        if (s->st) cudaStreamSynchronize(s->st);
        if (s->ev0) cudaEventDestroy(s->ev0);
        if (s->ev1) cudaEventDestroy(s->ev1);
        if (s->st) cudaStreamDestroy(s->st);
        delete s;
    }
    slots.clear();
    for (Lane *ln : lanes) {
        ln->ctx.destroy();
        if (ln->ev0) cudaEventDestroy(ln->ev0);
        if (ln->ev1) cudaEventDestroy(ln->ev1);
        delete ln;
    }
    lanes.clear();
    for (Ctx *c2 : fins) {
        c2->destroy();
        delete c2;
    }
    fins.clear();
    if (up) {
        cudaStreamSynchronize(up);
        cudaStreamDestroy(up);
    }
    if (up_ev) cudaEventDestroy(up_ev);
    if (epoch) cudaEventDestroy(epoch);
    up = nullptr;
    up_ev = epoch = nullptr;
    if (pool) cudaMemPoolDestroy(pool);
    pool = nullptr;
}

// ---- completion -------------------------------------------------------------------
void Server::complete_locked(Req *r, int status)
{
    dressx_server_request_t *p = r->pub;
    const Clock::time_point now = Clock::now();
    if (r->admitted) {
        reserved -= r->pl.bytes;
        --in_service;
    }
    p->status = status;
    p->path = r->pl.path;
    p->queue_ms = ms_between(r->t_submit, r->admitted ? r->t_admit : now);
    p->latency_ms = ms_between(r->t_submit, now);
    p->reserved_bytes = r->admitted ? r->pl.bytes : 0;
    if (status == DRESSX_OK) {
        ++completed;
        lat[r->cls].push_back(p->latency_ms);
        que[r->cls].push_back(p->queue_ms);
        fits += p->fits;
        edge_sweeps += p->edge_sweeps;
    } else if (status == DRESSX_ECANCELLED) {
        ++cancelled;
    } else {
        ++failed;
        ++cls_failed[r->cls];
    }
    live.erase(p);
    delete r;       // its device buffers were released by the worker
    std::atomic_thread_fence(std::memory_order_release);
    p->done = 1;
    wake = true;
    cv_done.notify_all();
    cv_sched.notify_one();
}

// A batch request whose slices have all run (or that stopped) goes to a
// finisher once no launch holds it.
void maybe_finish_locked(Server *sv, Req *r)
{
    if (!r->placed || r->queued_fin || r->inflight > 0) return;
    const bool stopped = r->cancelled || !r->err.ok();
    if (!stopped && r->items_done < r->pl.items) return;
    auto it = std::find(sv->active.begin(), sv->active.end(), r);
    if (it != sv->active.end()) sv->active.erase(it);
    r->queued_fin = true;
    sv->fin_q.push_back(r);
    sv->cv_fin.notify_one();
}

void Server::credit_locked(Slot *s)
{
    for (auto &c : s->credits) {
        Req *r = c.first;
        r->items_done += c.second;
        --r->inflight;
        if (!s->err.ok() && r->err.ok()) r->err = s->err;
        maybe_finish_locked(this, r);
    }
    s->credits.clear();
    s->busy = false;
    s->finished = false;
    s->err = Status::Ok();
    ++launches;
}

// ---- batch launches ---------------------------------------------------------------
// Launch geometry for requests of one class: group mode for whole-graph fits,
// CTA mode (parent staged in shared memory when that leaves enough groups)
// for subgraph fits.
bool geometry(BatchLaunch &L, bool plain, long long cap)
{
    if (plain) {
        L.per_group = 1;
        L.stage = 0;
        L.groups = std::max(1, 256 / L.gsize);
        while (L.groups > 1 && (long long)batch_smem_bytes(L) > cap) --L.groups;
        return (long long)batch_smem_bytes(L) <= cap;
    }
    L.per_group = 0;
    int tg = 512 / L.gsize;
    if (L.gsize > 32 && tg > 15) tg = 15;
    L.stage = 1;
    L.groups = tg;
    while (L.groups > 1 && (long long)batch_smem_bytes(L) > cap) --L.groups;
    if ((long long)batch_smem_bytes(L) > cap || L.groups * 2 < tg) {
        BatchLaunch L2 = L;
        L2.stage = 0;
        L2.groups = tg;
        while (L2.groups > 1 && (long long)batch_smem_bytes(L2) > cap) --L2.groups;
        if ((long long)batch_smem_bytes(L) > cap || L2.groups > L.groups) L = L2;
    }
    return (long long)batch_smem_bytes(L) <= cap;
}

bool Server::form_launch(Slot *s, BatchLaunch &L, std::vector<ParentDesc> &descs, std::vector<Chunk> &chunks)
{
    for (;;) {
        Req *first = nullptr;
        for (Req *r : active)
            if (!r->cancelled && r->err.ok() && r->next_item < r->pl.items) { first = r; break; }
        if (!first) return false;
        const bool plain = first->pl.item_kind == ITEM_PLAIN;
        const int gs = first->pl.gsize;
        std::vector<Req *> cand;
        for (Req *r : active)
            if (!r->cancelled && r->err.ok() && r->next_item < r->pl.items &&
                (r->pl.item_kind == ITEM_PLAIN) == plain && r->pl.gsize == gs)
                cand.push_back(r);
        auto shape = [&](const std::vector<Req *> &rs) {
            L = BatchLaunch{};
            L.gsize = gs;
            L.maxE = 1;
            L.maxN = 1;
            L.maxk = 1;
            L.M = 2;
            L.parent_bytes = 16;
            for (Req *r : rs) {
                L.maxE = std::max(L.maxE, r->pl.E);
                L.maxN = std::max(L.maxN, r->pl.N);
                L.maxk = std::max(L.maxk, r->pl.k);
                L.M = std::max(L.M, r->pl.M);
                L.parent_bytes = std::max(L.parent_bytes, r->pl.PL.bytes);
            }
            return geometry(L, plain, smem_cap);
        };
        if (!shape(cand)) {
            cand.assign(1, first);
            if (!shape(cand)) {
                first->err = Status::Err(DRESSX_EUNSUPPORTED, "fit state exceeds shared memory");
                maybe_finish_locked(this, first);
                continue;
            }
        }
        // every waiting request of the class gets a slice per round until the
        // launch holds launch_work edge-units
        const long long chunk_items = plain ? 1 : L.groups;
        std::unordered_map<Req *, int> idx;
        long long work = 0;
        bool progress = true;
        while (work < cfg.launch_work && progress) {
            progress = false;
            for (Req *r : cand) {
                if (r->next_item >= r->pl.items) continue;
                const long long n = std::min(chunk_items, r->pl.items - r->next_item);
                auto it = idx.find(r);
                int di;
                if (it == idx.end()) {
                    di = (int)descs.size();
                    idx[r] = di;
                    descs.push_back(r->desc);
                    s->credits.push_back({r, 0});
                    ++r->inflight;
                    r->started = true;
                } else {
                    di = it->second;
                }
                chunks.push_back({di, (int)n, r->next_item});
                r->next_item += n;
                s->credits[(size_t)di].second += n;
                work += n * std::max(1, r->pl.E);
                progress = true;
                if (work >= cfg.launch_work) break;
            }
        }
        active.erase(std::remove_if(active.begin(), active.end(),
                                    [](Req *r) { return r->next_item >= r->pl.items; }),
                     active.end());
        L.nchunks = (int)chunks.size();
        return true;
    }
}

Status Server::issue_launch(Slot *s, BatchLaunch &L, const std::vector<ParentDesc> &descs,
                            const std::vector<Chunk> &chunks)
{
    const size_t db = descs.size() * sizeof(ParentDesc), cb = chunks.size() * sizeof(Chunk);
    const size_t coff = (db + 255) & ~(size_t)255;
    const size_t kof = (coff + cb + 255) & ~(size_t)255;
    const size_t total = kof + 256;
    DRESS_TRY(s->host.reserve(kof));
    std::memcpy(s->host.ptr(), descs.data(), db);
    std::memcpy(s->host.ptr() + coff, chunks.data(), cb);
    if (s->dev.size() < total) DRESS_TRY(s->dev.alloc(total + total / 2, s->st));
    DRESS_CUDA_TRY(counted_memcpy(s->dev.get(), s->host.ptr(), coff + cb, cudaMemcpyHostToDevice, s->st));
    DRESS_CUDA_TRY(cudaMemsetAsync(s->dev.get() + kof, 0, sizeof(int), s->st));
    DRESS_CUDA_TRY(cudaStreamWaitEvent(s->st, up_ev, 0));     // the requests' uploads
    L.parents = (const ParentDesc *)s->dev.get();
    L.chunks = (const Chunk *)(s->dev.get() + coff);
    L.chunk_counter = (int *)(s->dev.get() + kof);
    DRESS_CUDA_TRY(cudaEventRecord(s->ev0, s->st));
    DRESS_TRY(launch_batch(L, sms, s->st));
    DRESS_CUDA_TRY(cudaEventRecord(s->ev1, s->st));
    DRESS_CUDA_TRY(cudaLaunchHostFunc(s->st, slot_done, s));
    return Status::Ok();
}

Status Server::admit_batch(Req *r)
{
    Planned &pl = r->pl;
    const size_t nvals = pl.item_kind == ITEM_PLAIN ? (size_t)pl.E + (size_t)pl.N : (size_t)pl.items * (size_t)pl.E;
    DRESS_TRY(r->d_data.alloc(pl.packed.size(), up));
    DRESS_TRY(r->d_values.alloc(std::max<size_t>(nvals, 1), up));
    DRESS_TRY(r->d_stats.alloc(ST_WORDS, up));
    DRESS_CUDA_TRY(counted_memcpy(r->d_data.get(), pl.packed.data(), pl.packed.size(), cudaMemcpyHostToDevice, up));
    DRESS_CUDA_TRY(cudaMemsetAsync(r->d_stats.get(), 0, ST_WORDS * sizeof(unsigned long long), up));
    DRESS_CUDA_TRY(cudaEventRecord(up_ev, up));
    std::vector<unsigned char>().swap(pl.packed);    // a pageable source is consumed on return
    ParentDesc &d = r->desc;
    d = ParentDesc{};
    d.N = pl.N;
    d.E = pl.E;
    d.S = pl.S;
    d.T = pl.T;
    d.kind = pl.item_kind;
    d.k = pl.k;
    d.fwd = pl.fwd;
    d.max_iter = r->pub->max_iterations;
    d.eps = r->pub->epsilon;
    d.has_nw = pl.has_nw;
    d.has_dinit = pl.has_dinit;
    d.data = r->d_data.get();
    d.values = (double *)r->d_values.get();
    d.stats = r->d_stats.get();
    d.multisets = nullptr;
    d.ranks = nullptr;
    d.offset = 0;
    d.stride = 1;
    return Status::Ok();
}

void Server::record_interval(cudaEvent_t a, cudaEvent_t b)
{
    float ta = 0.f, tb = 0.f;
    if (cudaEventElapsedTime(&ta, epoch, a) != cudaSuccess || cudaEventElapsedTime(&tb, epoch, b) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    std::lock_guard<std::mutex> lk(mu);
    if (intervals.size() >= (1u << 20)) intervals.erase(intervals.begin(), intervals.begin() + (1 << 19));
    intervals.push_back({(double)ta, (double)tb});
}

void Server::scheduler()
{
    cudaSetDevice(device);
    tls_pool = pool;
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
        // admission in arrival order: the head waits until its bytes fit
        std::vector<Req *> adm;
        while (!waiting.empty()) {
            Req *r = waiting.front();
            if (reserved + r->pl.bytes > budget) break;
            waiting.pop_front();
            r->admitted = true;
            r->t_admit = Clock::now();
            reserved += r->pl.bytes;
            peak_reserved = std::max(peak_reserved, reserved);
            ++in_service;
            max_in_service = std::max(max_in_service, in_service);
            adm.push_back(r);
        }
        std::vector<Slot *> done;
        for (Slot *s : slots)
            if (s->busy && s->finished) done.push_back(s);
        lk.unlock();
        for (Req *r : adm)
            if (r->pl.path == DRESSX_PATH_BATCH) {
                r->err = admit_batch(r);
                if (!r->err.ok()) set_last_error(r->err);
            }
        for (Slot *s : done) record_interval(s->ev0, s->ev1);
        lk.lock();
        for (Req *r : adm) {
            r->placed = true;
            if (r->pl.path == DRESSX_PATH_LANE) {
                lane_q.push_back(r);
                cv_lane.notify_one();
            } else if (!r->err.ok() || r->cancelled) {
                r->queued_fin = true;
                fin_q.push_back(r);
                cv_fin.notify_one();
            } else {
                active.push_back(r);
            }
        }
        for (Slot *s : done) credit_locked(s);
        for (;;) {
            Slot *slot = nullptr;
            for (Slot *s : slots)
                if (!s->busy) { slot = s; break; }
            if (!slot) break;
            BatchLaunch L{};
            std::vector<ParentDesc> descs;
            std::vector<Chunk> chunks;
            if (!form_launch(slot, L, descs, chunks)) break;
            slot->busy = true;
            slot->finished = false;
            lk.unlock();
            Status st = issue_launch(slot, L, descs, chunks);
            if (!st.ok()) cudaStreamSynchronize(slot->st);   // whatever was enqueued is done before reuse
            lk.lock();
            if (!st.ok()) {             // nothing will report this launch: fail its requests now
                set_last_error(st);
                slot->err = st;
                slot->finished = true;
                wake = true;
            }
        }
        if (stop) break;
        cv_sched.wait_for(lk, std::chrono::milliseconds(20), [&] { return wake; });
        wake = false;
    }
}

// ---- finishers and lanes ---------------------------------------------------------
Status collect_batch(Server *sv, Req *r, Ctx *ctx)
{
    dressx_server_request_t *p = r->pub;
    const Planned &pl = r->pl;
    unsigned long long st[ST_WORDS];
    DRESS_CUDA_TRY(counted_memcpy(st, r->d_stats.get(), sizeof st, cudaMemcpyDeviceToHost, ctx->st));
    DRESS_CUDA_TRY(cudaStreamSynchronize(ctx->st));
    if (pl.item_kind == ITEM_PLAIN) {
        p_dress_graph_t g = p->graph;
        if (pl.E)
            DRESS_CUDA_TRY(counted_memcpy(g->edge_dress, r->d_values.get(), (size_t)pl.E * sizeof(double),
                                           cudaMemcpyDeviceToHost, ctx->st));
        if (st[ST_SWEEPS] > 0 && pl.N)
            DRESS_CUDA_TRY(counted_memcpy(g->vertex_dress, (double *)r->d_values.get() + pl.E,
                                           (size_t)pl.N * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
        DRESS_CUDA_TRY(cudaStreamSynchronize(ctx->st));
        p->iterations = (int)(long long)st[ST_ITERATIONS];
        if (st[ST_SWEEPS] > 0) std::memcpy(&p->delta, &st[ST_DELTA], sizeof(double));
        p->fits = 1;
        p->edge_sweeps = (int64_t)st[ST_EDGE_ITERS];
        return Status::Ok();
    }
    p->num_subgraphs = pl.num_subgraphs;
    p->fits = (int64_t)st[ST_FITS];
    p->edge_sweeps = (int64_t)st[ST_EDGE_ITERS];
    const long long n = (long long)st[ST_CURSOR];
    if (n <= 0) return Status::Ok();
    // the histogram straight into its malloc'd array, through this
    // finisher's pinned stage
    DevBuf<unsigned long long> alt;
    DRESS_TRY(alt.alloc((size_t)n, ctx->st));
    HistResult res;
    DRESS_TRY(histogram_device(r->d_values.get(), alt.get(), std::vector<long long>{0}, std::vector<long long>{n}, res,
                               ctx->st, sv->sms));
    std::vector<int64_t *> outs;
    std::vector<long long> lens;
    // at most 8 copy threads: lanes and other finishers share the host
    DRESS_TRY(histogram_fetch(res, outs, lens, ctx->stage, ctx->st, sv->sms, nullptr, nullptr, 8));
    p->hist_flat = outs[0];
    p->hist_len = (int)lens[0];
    return Status::Ok();
}

void Server::fin_main(Ctx *ctx)
{
    cudaSetDevice(device);
    tls_pool = pool;
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
        cv_fin.wait(lk, [&] { return stop || !fin_q.empty(); });
        if (fin_q.empty()) {
            if (stop) break;
            continue;
        }
        Req *r = fin_q.front();
        fin_q.pop_front();
        lk.unlock();
        int status = DRESSX_OK;
        if (!r->err.ok()) {
            status = r->err.code;
        } else if (r->cancelled) {
            status = DRESSX_ECANCELLED;
        } else {
            Status s = collect_batch(this, r, ctx);
            if (!s.ok()) {
                set_last_error(s);
                status = s.code;
            }
        }
        cudaStreamSynchronize(ctx->st);
        r->d_data.release();
        r->d_values.release();
        r->d_stats.release();
        lk.lock();
        complete_locked(r, status);
    }
}

int run_lane(Server *sv, Req *r, Lane *ln)
{
    dressx_server_request_t *p = r->pub;
    cudaEventRecord(ln->ev0, ln->ctx.st);
    Status s;
    if (p->kind == DRESSX_FIT) {
        int it = p->iterations;
        double dl = p->delta;
        FitStats fs;
        s = fit_graph(p->graph, p->max_iterations, p->epsilon, &it, &dl, &fs, ln->ctx);
        if (s.ok()) {
            p->iterations = it;
            p->delta = dl;
            p->fits = 1;
            p->edge_sweeps = (int64_t)fs.sweeps * p->graph->E;
        }
    } else {
        dressx_hist_request_t hr{};
        hr.graph = p->graph;
        hr.kind = p->kind;
        hr.k = p->k;
        hr.max_iterations = p->max_iterations;
        hr.epsilon = p->epsilon;
        hr.offset = 0;
        hr.stride = 1;
        hr.want_histogram = 1;
        int64_t es = 0;
        s = hist_batch_core(&hr, 1, false, ln->ctx, &es);
        if (s.ok() && hr.status != DRESSX_OK) s = Status::Err(hr.status, "Delta/Nabla request failed");
        p->hist_flat = hr.hist_flat;
        p->hist_len = hr.hist_len;
        p->num_subgraphs = hr.num_subgraphs;
        p->fits = hr.fits;
        p->edge_sweeps = es;
    }
    cudaEventRecord(ln->ev1, ln->ctx.st);
    cudaStreamSynchronize(ln->ctx.st);
    sv->record_interval(ln->ev0, ln->ev1);
    if (!s.ok()) set_last_error(s);
    return s.code;
}

void Server::lane_main(Lane *ln)
{
    cudaSetDevice(device);
    tls_pool = pool;
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
        cv_lane.wait(lk, [&] { return stop || !lane_q.empty(); });
        if (lane_q.empty()) {
            if (stop) break;
            continue;
        }
        Req *r = lane_q.front();
        lane_q.pop_front();
        r->started = true;
        lk.unlock();
        int status = run_lane(this, r, ln);
        lk.lock();
        complete_locked(r, status);
    }
}

// nearest-rank quantile of an unsorted sample
double quantile(std::vector<double> v, double q)
{
    if (v.empty()) return 0.0;
    size_t i = (size_t)std::ceil(q * (double)v.size());
    i = i == 0 ? 0 : i - 1;
    if (i >= v.size()) i = v.size() - 1;
    std::nth_element(v.begin(), v.begin() + (long)i, v.end());
    return v[i];
}

}  // namespace
}  // namespace dress

using namespace dress;

struct dressx_server {
    Server s;
};

extern "C" {

int dressx_server_create(const dressx_server_config_t *cfg, dressx_server_t **out)
{
    if (!out) return DRESSX_EINVAL;
    *out = nullptr;
    dressx_server *sv = new dressx_server;
    Status s = sv->s.start(cfg);
    if (!s.ok()) {
        set_last_error(s);
        sv->s.shutdown();
        delete sv;
        return s.code;
    }
    *out = sv;
    return DRESSX_OK;
}

int dressx_server_submit(dressx_server_t *h, dressx_server_request_t *p)
{
    if (!h || !p) return DRESSX_EINVAL;
    Server &sv = h->s;
    {
        std::lock_guard<std::mutex> lk(sv.mu);
        if (sv.live.count(p)) return DRESSX_EINVAL;     // still in service: leave it untouched
    }
    p->done = 0;
    p->status = DRESSX_OK;
    p->hist_flat = nullptr;
    p->hist_len = 0;
    p->num_subgraphs = 0;
    p->fits = 0;
    p->edge_sweeps = 0;
    p->path = DRESSX_PATH_NONE;
    p->queue_ms = p->latency_ms = 0.0;
    p->reserved_bytes = 0;
    Req *r = new Req;
    r->pub = p;
    r->t_submit = Clock::now();
    Status s = plan_request(p->graph, p->kind, p->k, sv.smem_cap, true, r->pl);
    if (s.ok() && r->pl.bytes > sv.budget)
        s = Status::Err(DRESSX_EBUDGET, "request needs " + std::to_string(r->pl.bytes) +
                                        " device bytes, more than the budget");
    r->cls = class_of(p->kind, r->pl.path);
    std::unique_lock<std::mutex> lk(sv.mu);
    if (s.ok() && sv.closing) s = Status::Err(DRESSX_ECANCELLED, "server is shutting down");
    if (s.ok() && (long long)sv.waiting.size() >= sv.cfg.max_queued) s = Status::Err(DRESSX_EBUSY, "queue full");
    if (s.ok() && sv.live.count(p)) s = Status::Err(DRESSX_EINVAL, "request already in service");
    ++sv.submitted;
    if (!s.ok()) {
        ++sv.rejected;
        p->status = s.code;
        p->path = r->pl.path;
        delete r;
        lk.unlock();
        set_last_error(s);
        std::atomic_thread_fence(std::memory_order_release);
        p->done = 1;
        return s.code;
    }
    r->seq = sv.seq++;
    sv.live[p] = r;
    sv.waiting.push_back(r);
    sv.wake = true;
    sv.cv_sched.notify_one();
    return DRESSX_OK;
}

int dressx_server_wait(dressx_server_t *h, dressx_server_request_t *p, int timeout_ms)
{
    if (!h || !p) return DRESSX_EINVAL;
    Server &sv = h->s;
    std::unique_lock<std::mutex> lk(sv.mu);
    auto ready = [&] { return p->done != 0; };
    if (timeout_ms < 0) sv.cv_done.wait(lk, ready);
    else if (!sv.cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) return DRESSX_ETIMEOUT;
    return p->status;
}

int dressx_server_cancel(dressx_server_t *h, dressx_server_request_t *p)
{
    if (!h || !p) return DRESSX_EINVAL;
    Server &sv = h->s;
    std::lock_guard<std::mutex> lk(sv.mu);
    auto it = sv.live.find(p);
    if (it == sv.live.end()) return p->done ? DRESSX_EBUSY : DRESSX_EINVAL;
    Req *r = it->second;
    if (!r->admitted) {
        sv.waiting.erase(std::find(sv.waiting.begin(), sv.waiting.end(), r));
        sv.complete_locked(r, DRESSX_ECANCELLED);
        return DRESSX_OK;
    }
    if (r->pl.path == DRESSX_PATH_LANE) {
        auto q = std::find(sv.lane_q.begin(), sv.lane_q.end(), r);
        if (q == sv.lane_q.end()) return DRESSX_EBUSY;
        sv.lane_q.erase(q);
        sv.complete_locked(r, DRESSX_ECANCELLED);
        return DRESSX_OK;
    }
    if (r->cancelled) return DRESSX_OK;
    if (r->queued_fin || r->next_item >= r->pl.items) return DRESSX_EBUSY;
    r->cancelled = true;
    maybe_finish_locked(&sv, r);
    return DRESSX_OK;
}

int dressx_server_drain(dressx_server_t *h, int timeout_ms)
{
    if (!h) return DRESSX_EINVAL;
    Server &sv = h->s;
    std::unique_lock<std::mutex> lk(sv.mu);
    auto idle = [&] { return sv.live.empty(); };
    if (timeout_ms < 0) sv.cv_done.wait(lk, idle);
    else if (!sv.cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), idle)) return DRESSX_ETIMEOUT;
    return DRESSX_OK;
}

int dressx_server_stats(dressx_server_t *h, dressx_server_stats_t *out, int reset)
{
    if (!h || !out) return DRESSX_EINVAL;
    Server &sv = h->s;
    unsigned long long pool_bytes = 0;
    if (sv.pool) cudaMemPoolGetAttribute(sv.pool, cudaMemPoolAttrReservedMemCurrent, &pool_bytes);
    std::lock_guard<std::mutex> lk(sv.mu);
    std::memset(out, 0, sizeof *out);
    out->elapsed_s = ms_between(sv.t0, Clock::now()) / 1e3;
    out->submitted = sv.submitted;
    out->completed = sv.completed;
    out->failed = sv.failed;
    out->cancelled = sv.cancelled;
    out->rejected = sv.rejected;
    out->fits = sv.fits;
    out->edge_sweeps = sv.edge_sweeps;
    out->batch_launches = sv.launches;
    out->budget_bytes = sv.budget;
    out->reserved_bytes = sv.reserved;
    out->peak_reserved_bytes = sv.peak_reserved;
    out->pool_bytes = (int64_t)pool_bytes;
    out->max_in_service = sv.max_in_service;
    std::vector<std::pair<double, double>> iv = sv.intervals;
    std::sort(iv.begin(), iv.end());
    double busy = 0.0, work = 0.0, cs = 0.0, ce = -1.0;
    for (auto &x : iv) {
        work += x.second - x.first;
        if (x.first > ce) {
            if (ce > cs) busy += ce - cs;
            cs = x.first;
            ce = x.second;
        } else if (x.second > ce) {
            ce = x.second;
        }
    }
    if (ce > cs) busy += ce - cs;
    out->device_busy_ms = busy;
    out->device_work_ms = work;
    for (int c = 0; c < DRESSX_CLASSES; ++c) {
        dressx_server_class_stats_t &o = out->cls[c];
        const std::vector<double> &v = sv.lat[c];
        o.completed = (int64_t)v.size();
        o.failed = sv.cls_failed[c];
        o.p50_ms = quantile(v, 0.50);
        o.p99_ms = quantile(v, 0.99);
        double sum = 0.0, mx = 0.0;
        for (double x : v) {
            sum += x;
            mx = std::max(mx, x);
        }
        o.mean_ms = v.empty() ? 0.0 : sum / (double)v.size();
        o.max_ms = mx;
        o.queue_p50_ms = quantile(sv.que[c], 0.50);
        o.queue_p99_ms = quantile(sv.que[c], 0.99);
    }
    if (reset) {
        sv.t0 = Clock::now();
        sv.submitted = sv.completed = sv.failed = sv.cancelled = sv.rejected = 0;
        sv.fits = sv.edge_sweeps = sv.launches = 0;
        sv.peak_reserved = sv.reserved;
        sv.max_in_service = sv.in_service;
        for (int c = 0; c < DRESSX_CLASSES; ++c) {
            sv.lat[c].clear();
            sv.que[c].clear();
            sv.cls_failed[c] = 0;
        }
        sv.intervals.clear();
    }
    return DRESSX_OK;
}

int dressx_server_destroy(dressx_server_t *h)
{
    if (!h) return DRESSX_EINVAL;
    h->s.shutdown();
    delete h;
    return DRESSX_OK;
}

int dressx_server_estimate(p_dress_graph_t g, int kind, int k, int64_t *bytes, int *path)
{
    Planned pl;
    Status s = plan_request(g, kind, k, B200_SMEM_OPTIN - 256, false, pl);
    if (!s.ok()) {
        set_last_error(s);
        return s.code;
    }
    if (bytes) *bytes = pl.bytes;
    if (path) *path = pl.path;
    return DRESSX_OK;
}

}  // extern "C"
