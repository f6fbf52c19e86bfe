// engine.cpp -- process-wide engine state and the fit entry points.
//
// One engine per process: a non-blocking stream on the device that was
// current at first use (or dressx_config_t.device), a side stream, and the
// device's default memory pool with a high release threshold so buffers are
// recycled between calls instead of returned to the driver.  Legacy entry
// points are serialised by a mutex; none of them calls exit().
#include <cstdio>
#include <cstring>
#include <cstdint>
#include <emmintrin.h>
#include <mutex>

#include <algorithm>

#include "engine.h"
#include "host_par.h"

namespace dress {

namespace {
std::mutex g_err_mu;
int g_err_code = DRESSX_OK;
std::string g_err_msg;
FitStats g_last_stats;
}  // namespace

void set_last_error(const Status &s)
{
    std::lock_guard<std::mutex> lk(g_err_mu);
    g_err_code = s.code;
    g_err_msg = s.msg;
    if (!s.ok()) std::fprintf(stderr, "dress_b200: %s\n", s.msg.c_str());
}

Pinned::~Pinned()
{
    if (base_) cudaFreeHost(base_);
    for (char *r : retired_) cudaFreeHost(r);
}

Status Pinned::reserve(size_t bytes)
{
    if (bytes <= cap_) return Status::Ok();
    // Pinning host memory is slow, so the buffer grows at least twofold (and
    // to at least 32 MiB): a stream of growing requests reallocates it a few
    // times, not at every request.  Freeing pinned memory waits for the whole
    // device -- every stream of every lane -- so an outgrown buffer is kept
    // until the owner goes away (at most the final size again, the growth
    // being geometric); only when pinning fails are the old buffers freed
    // and the allocation retried.
    const size_t want = std::max(bytes, std::max(2 * cap_, (size_t)32 << 20));
    char *nb = nullptr;
    if (cudaMallocHost((void **)&nb, want) != cudaSuccess) {
        cudaGetLastError();
        nb = nullptr;
        if (base_) cudaFreeHost(base_);
        for (char *r : retired_) cudaFreeHost(r);
        retired_.clear();
        base_ = nullptr;
        cap_ = 0;
        if (cudaMallocHost((void **)&nb, bytes) != cudaSuccess) {
            cudaGetLastError();
            return Status::Err(DRESSX_ENOMEM, "pinned host allocation failed");
        }
        base_ = nb;
        cap_ = bytes;
        return Status::Ok();
    }
    if (base_) retired_.push_back(base_);
    base_ = nb;
    cap_ = want;
    return Status::Ok();
}

// ---- staged copies ----------------------------------------------------------
void copy_nt(void *dst, const void *src, size_t n)
{
    char *d = (char *)dst;
    const char *s = (const char *)src;
    if (n < 4096) {
        std::memcpy(d, s, n);
        return;
    }
    const size_t head = (16 - ((uintptr_t)d & 15)) & 15;
    std::memcpy(d, s, head);
    d += head;
    s += head;
    n -= head;
    const size_t body = n & ~(size_t)63;
    __m128i *dv = (__m128i *)d;
    if (((uintptr_t)s & 15) == 0) {
        const __m128i *sv = (const __m128i *)s;
        for (size_t i = 0; i < body / 16; i += 4) {
            const __m128i x0 = _mm_load_si128(sv + i), x1 = _mm_load_si128(sv + i + 1);
            const __m128i x2 = _mm_load_si128(sv + i + 2), x3 = _mm_load_si128(sv + i + 3);
            _mm_stream_si128(dv + i, x0);
            _mm_stream_si128(dv + i + 1, x1);
            _mm_stream_si128(dv + i + 2, x2);
            _mm_stream_si128(dv + i + 3, x3);
        }
    } else {
        const __m128i *sv = (const __m128i *)s;
        for (size_t i = 0; i < body / 16; i += 4) {
            const __m128i x0 = _mm_loadu_si128(sv + i), x1 = _mm_loadu_si128(sv + i + 1);
            const __m128i x2 = _mm_loadu_si128(sv + i + 2), x3 = _mm_loadu_si128(sv + i + 3);
            _mm_stream_si128(dv + i, x0);
            _mm_stream_si128(dv + i + 1, x1);
            _mm_stream_si128(dv + i + 2, x2);
            _mm_stream_si128(dv + i + 3, x3);
        }
    }
    _mm_sfence();
    std::memcpy(d + body, s + body, n - body);
}

namespace {

// Pieces of the byte range [lo, hi) of the spans taken as one range, in span
// order: fn(span, offset in the span, length, offset from lo).
template <class F>
void for_pieces(const HostSpan *spans, int n, size_t lo, size_t hi, F fn)
{
    size_t base = 0;
    for (int i = 0; i < n && base < hi; ++i) {
        const size_t b = std::max(lo, base), e = std::min(hi, base + spans[i].bytes);
        if (b < e) fn(spans[i], b - base, e - b, b - lo);
        base += spans[i].bytes;
    }
}

// host copy of chunk k between its stage slot and the spans, split over
// host threads in 2 MiB grains
void host_part(const HostSpan *spans, int n, char *stage, size_t k, size_t total, bool to_stage)
{
    constexpr size_t grain = (size_t)2 << 20;
    char *slot = stage + (k & 1) * STAGE_CHUNK;
    const size_t lo = k * STAGE_CHUNK, hi = std::min(total, lo + STAGE_CHUNK);
    const long long pieces = (long long)((hi - lo + grain - 1) / grain);
    parallel_for(pieces, host_threads(pieces), [&](long long g) {
        const size_t a = lo + (size_t)g * grain, b = std::min(hi, a + grain);
        for_pieces(spans, n, a, b, [&](const HostSpan &sp, size_t off, size_t len, size_t at) {
            char *st = slot + (a - lo) + at;
            if (to_stage) copy_nt(st, (const char *)sp.host + off, len);
            else copy_nt((char *)sp.host + off, st, len);
        });
    });
}

Status staged_copy(const HostSpan *spans, int n, Pinned *pin, cudaStream_t cs, bool up)
{
    size_t total = 0;
    for (int i = 0; i < n; ++i) total += spans[i].bytes;
    if (total == 0) return Status::Ok();
    if (total <= ((size_t)1 << 20) || !pin) {
        // small copies: the driver's own staging is as quick
        for (int i = 0; i < n; ++i) {
            if (!spans[i].bytes) continue;
            if (up) DRESS_CUDA_TRY(counted_memcpy(spans[i].dev, spans[i].host, spans[i].bytes, cudaMemcpyHostToDevice, cs));
            else DRESS_CUDA_TRY(counted_memcpy(spans[i].host, spans[i].dev, spans[i].bytes, cudaMemcpyDeviceToHost, cs));
        }
        DRESS_CUDA_TRY(cudaStreamSynchronize(cs));
        return Status::Ok();
    }
    DRESS_TRY(pin->reserve(2 * STAGE_CHUNK));
    char *stage = pin->ptr();
    cudaEvent_t ev[2] = {nullptr, nullptr};
    for (auto &e : ev) DRESS_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    struct EvGuard {
        cudaEvent_t *e;
        ~EvGuard()
        {
            cudaEventSynchronize(e[0]);
            cudaEventSynchronize(e[1]);
            cudaEventDestroy(e[0]);
            cudaEventDestroy(e[1]);
        }
    } guard{ev};
    const size_t nchunks = (total + STAGE_CHUNK - 1) / STAGE_CHUNK;
    for (size_t k = 0; k < nchunks; ++k) {
        char *slot = stage + (k & 1) * STAGE_CHUNK;
        const size_t lo = k * STAGE_CHUNK, hi = std::min(total, lo + STAGE_CHUNK);
        if (k >= 2) DRESS_CUDA_TRY(cudaEventSynchronize(ev[k & 1]));     // the slot's last copy is done
        if (up) host_part(spans, n, stage, k, total, true);
        Status err;
        for_pieces(spans, n, lo, hi, [&](const HostSpan &sp, size_t off, size_t len, size_t at) {
            cudaError_t e = up ? cudaMemcpyAsync((char *)sp.dev + off, slot + at, len, cudaMemcpyHostToDevice, cs)
                               : cudaMemcpyAsync(slot + at, (const char *)sp.dev + off, len, cudaMemcpyDeviceToHost,
                                                 cs);
            if (e != cudaSuccess && err.ok()) err = Status::Err(DRESSX_ECUDA, cudaGetErrorString(e));
        });
        DRESS_TRY(err);
        if (up) count_h2d(hi - lo);
        else count_d2h(hi - lo);
        DRESS_CUDA_TRY(cudaEventRecord(ev[k & 1], cs));
        if (!up && k >= 1) {
            // the previous chunk is on the host: copy it out while this one is in flight
            DRESS_CUDA_TRY(cudaEventSynchronize(ev[(k - 1) & 1]));
            host_part(spans, n, stage, k - 1, total, false);
        }
    }
    if (!up) {
        DRESS_CUDA_TRY(cudaEventSynchronize(ev[(nchunks - 1) & 1]));
        host_part(spans, n, stage, nchunks - 1, total, false);
    }
    return Status::Ok();
}

}  // namespace

Status staged_upload(const HostSpan *spans, int n, const Ctx &ctx)
{
    return staged_copy(spans, n, ctx.stage, ctx.st, true);
}
Status staged_download(const HostSpan *spans, int n, const Ctx &ctx)
{
    return staged_copy(spans, n, ctx.stage, ctx.st, false);
}
Status staged_upload_via(const HostSpan *spans, int n, Pinned *stage, cudaStream_t st)
{
    return staged_copy(spans, n, stage, st, true);
}

thread_local cudaMemPool_t tls_pool = nullptr;
thread_local long long tls_launches = 0;

Status Ctx::create(int dev, int sms, const dressx_config_t *config, int priority)
{
    device = dev;
    num_sms = sms;
    cfg = config;
    DRESS_CUDA_TRY(cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, priority));
    DRESS_CUDA_TRY(cudaStreamCreateWithPriority(&side, cudaStreamNonBlocking, priority));
    DRESS_CUDA_TRY(cudaStreamCreateWithPriority(&side2, cudaStreamNonBlocking, priority));
    DRESS_CUDA_TRY(cudaStreamCreateWithPriority(&side3, cudaStreamNonBlocking, priority));
    DRESS_CUDA_TRY(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    DRESS_CUDA_TRY(cudaEventCreateWithFlags(&join, cudaEventDisableTiming));
    DRESS_CUDA_TRY(cudaEventCreateWithFlags(&join2, cudaEventDisableTiming));
    DRESS_CUDA_TRY(cudaEventCreateWithFlags(&join3, cudaEventDisableTiming));
    stage = new Pinned();
    stage2 = new Pinned();
    return Status::Ok();
}

void Ctx::destroy()
{
    if (st) cudaStreamSynchronize(st);
    if (side) cudaStreamSynchronize(side);
    if (side2) cudaStreamSynchronize(side2);
    if (side3) cudaStreamSynchronize(side3);
    if (fork) cudaEventDestroy(fork);
    if (join) cudaEventDestroy(join);
    if (join2) cudaEventDestroy(join2);
    if (join3) cudaEventDestroy(join3);
    if (st) cudaStreamDestroy(st);
    if (side) cudaStreamDestroy(side);
    if (side2) cudaStreamDestroy(side2);
    if (side3) cudaStreamDestroy(side3);
    st = side = side2 = side3 = nullptr;
    fork = join = join2 = join3 = nullptr;
    delete stage;
    stage = nullptr;
    delete stage2;
    stage2 = nullptr;
}

Status Engine::init()
{
    if (ctx.st) return Status::Ok();
    int dev = cfg.device;
    if (dev < 0) DRESS_CUDA_TRY(cudaGetDevice(&dev));
    DRESS_CUDA_TRY(cudaSetDevice(dev));
    device = dev;
    DRESS_CUDA_TRY(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev));
    DRESS_TRY(ctx.create(dev, num_sms, &cfg));
    cudaMemPool_t pool;
    DRESS_CUDA_TRY(cudaDeviceGetDefaultMemPool(&pool, dev));
    unsigned long long keep = cfg.memory_budget_bytes ? cfg.memory_budget_bytes : ~0ULL;
    DRESS_CUDA_TRY(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    return Status::Ok();
}

Engine &engine()
{
    static Engine e;
    return e;
}

Status fit_locked(p_dress_graph_t g, int max_iterations, double epsilon, int *iterations, double *delta)
{
    Engine &en = engine();
    std::lock_guard<std::mutex> lk(en.mu);
    DRESS_TRY(en.init());
    DRESS_CUDA_TRY(cudaSetDevice(en.device));
    FitStats st;
    Status s = fit_graph(g, max_iterations, epsilon, iterations, delta, &st, en.ctx);
    if (s.ok()) g_last_stats = st;
    return s;
}

}  // namespace dress

using namespace dress;

extern "C" {

int dressx_configure(const dressx_config_t *cfg)
{
    Engine &en = engine();
    std::lock_guard<std::mutex> lk(en.mu);
    if (!cfg) return DRESSX_EINVAL;
    if (en.ctx.st && cfg->device >= 0 && cfg->device != en.device) {
        set_last_error(Status::Err(DRESSX_EINVAL, "engine already bound to another device"));
        return DRESSX_EINVAL;
    }
    en.cfg = *cfg;
    return DRESSX_OK;
}

int dressx_last_error(char *msg, int msg_len)
{
    std::lock_guard<std::mutex> lk(g_err_mu);
    if (msg && msg_len > 0) {
        std::strncpy(msg, g_err_msg.c_str(), (size_t)msg_len - 1);
        msg[msg_len - 1] = 0;
    }
    return g_err_code;
}

int dressx_fit(p_dress_graph_t g, int max_iterations, double epsilon, int *iterations, double *delta)
{
    Status s = fit_locked(g, max_iterations, epsilon, iterations, delta);
    set_last_error(s);
    return s.code;
}

int dressx_last_fit_stats(dressx_fit_stats_t *out)
{
    if (!out) return DRESSX_EINVAL;
    out->common_terms = g_last_stats.T;
    out->sweeps = g_last_stats.sweeps;
    out->setup_ms = g_last_stats.setup_ms;
    out->iterate_ms = g_last_stats.iterate_ms;
    for (int b = 0; b < 8; ++b) {
        out->vertex_bin_items[b] = g_last_stats.vbin_items[b];
        out->vertex_bin_terms[b] = g_last_stats.vbin_terms[b];
        out->edge_bin_items[b] = g_last_stats.ebin_items[b];
        out->edge_bin_terms[b] = g_last_stats.ebin_terms[b];
    }
    for (int i = 0; i < 5; ++i) out->phase_ms[i] = g_last_stats.phase_ms[i];
    return DRESSX_OK;
}

void dress_fit_cuda(p_dress_graph_t g, int max_iterations, double epsilon, int *iterations, double *delta)
{
    dressx_fit(g, max_iterations, epsilon, iterations, delta);
}

void dress_fit(p_dress_graph_t g, int max_iterations, double epsilon, int *iterations, double *delta)
{
    dressx_fit(g, max_iterations, epsilon, iterations, delta);
}

void dressx_free(void *p) { free(p); }

int dressx_stream(void **stream)
{
    if (!stream) return DRESSX_EINVAL;
    Engine &en = engine();
    std::lock_guard<std::mutex> lk(en.mu);
    Status s = en.init();
    set_last_error(s);
    *stream = s.ok() ? (void *)en.ctx.st : nullptr;
    return s.code;
}

int dressx_counters(int64_t *h2d_bytes, int64_t *d2h_bytes, int64_t *launches, int reset)
{
    Engine &en = engine();
    std::lock_guard<std::mutex> lk(en.mu);
    if (h2d_bytes) *h2d_bytes = en.h2d_bytes.load();
    if (d2h_bytes) *d2h_bytes = en.d2h_bytes.load();
    if (launches) *launches = en.launches.load();
    if (reset) {
        en.h2d_bytes = 0;
        en.d2h_bytes = 0;
        en.launches = 0;
    }
    return DRESSX_OK;
}

}  // extern "C"
