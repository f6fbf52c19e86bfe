// engine.h -- internal C++ interface of the B200 DRESS engine.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>
#include <atomic>
#include <mutex>
#include <string>
#include <vector>

#include "dress_b200.h"
#include "dress_b200_ext.h"

namespace dress {

// ---- status ------------------------------------------------------------
struct Status {
    int code = DRESSX_OK;
    std::string msg;
    bool ok() const { return code == DRESSX_OK; }
    static Status Ok() { return Status(); }
    static Status Err(int c, const std::string &m) { Status s; s.code = c; s.msg = m; return s; }
};

#define DRESS_CUDA_TRY(call)                                                   \
    do {                                                                       \
        cudaError_t _e = (call);                                               \
        if (_e != cudaSuccess)                                                 \
            return ::dress::Status::Err(DRESSX_ECUDA,                          \
                std::string(#call) + ": " + cudaGetErrorString(_e));           \
    } while (0)

#define DRESS_TRY(expr)                                                        \
    do {                                                                       \
        ::dress::Status _s = (expr);                                           \
        if (!_s.ok()) return _s;                                               \
    } while (0)

// ---- stream-ordered device buffers -------------------------------------
// Device memory comes from a stream-ordered memory pool: the device's
// default pool (release threshold = the configured budget), or, on threads
// that set tls_pool, that pool -- a request server points its worker threads
// at its own arena pool, so every buffer of a served request is drawn from
// the server's resident memory.  Freed blocks stay in the pool, so repeated
// work of the same size allocates nothing from the driver after the first.
extern thread_local cudaMemPool_t tls_pool;

template <class T>
class DevBuf {
  public:
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    Status alloc(size_t n, cudaStream_t st)
    {
        release();
        st_ = st;
        n_ = n;
        if (n == 0) return Status::Ok();
        cudaError_t e = tls_pool ? cudaMallocFromPoolAsync((void **)&p_, n * sizeof(T), tls_pool, st)
                                 : cudaMallocAsync((void **)&p_, n * sizeof(T), st);
        if (e != cudaSuccess) {
            p_ = nullptr;
            cudaGetLastError();
            return Status::Err(DRESSX_ENOMEM, "device allocation of " +
                               std::to_string(n * sizeof(T)) + " bytes failed");
        }
        return Status::Ok();
    }
    void release()
    {
        if (p_) cudaFreeAsync(p_, st_);
        p_ = nullptr;
        n_ = 0;
    }
    T *get() const { return p_; }
    size_t size() const { return n_; }
  private:
    T *p_ = nullptr;
    size_t n_ = 0;
    cudaStream_t st_ = nullptr;
};

// ---- pinned host staging buffer ------------------------------------------
class Pinned {
  public:
    ~Pinned();
    Status reserve(size_t bytes);
    char *ptr() { return base_; }
  private:
    char *base_ = nullptr;
    size_t cap_ = 0;
    std::vector<char *> retired_;          // outgrown buffers, freed with the owner
};

// ---- an execution context: where one stream of work runs ------------------
// The legacy entry points share the engine's context; every server lane owns
// one, so lanes keep independent work in flight on the device at once.
struct Ctx {
    int device = 0;
    int num_sms = 148;
    cudaStream_t st = nullptr;             // main stream
    cudaStream_t side = nullptr;           // concurrent hub work of the single-graph fit
    cudaStream_t side2 = nullptr;          // ... and its block items below the hubs
    cudaStream_t side3 = nullptr;          // ... and its thread-per-item bins
    cudaEvent_t fork = nullptr, join = nullptr, join2 = nullptr, join3 = nullptr;
    const dressx_config_t *cfg = nullptr;
    Pinned *stage = nullptr;               // host staging of this context's uploads and downloads
    Pinned *stage2 = nullptr;              // a second stage: an upload on a host thread of its own
    // priority: CUDA stream priority of both streams (0 = default; lower
    // numbers are served first by the block scheduler)
    Status create(int dev, int sms, const dressx_config_t *config, int priority = 0);
    void destroy();
};

// ---- the per-process engine ------------------------------------------------
struct Engine {
    int device = -1;
    Ctx ctx;                               // context of the legacy entry points
    std::mutex mu;                         // legacy entry points are serialised
    int num_sms = 148;
    dressx_config_t cfg;
    // traffic and launch counters of the public calls (reset by the caller)
    std::atomic<long long> h2d_bytes{0}, d2h_bytes{0}, launches{0};
    Status init();
};

Engine &engine();
void set_last_error(const Status &s);

inline void count_h2d(size_t b) { engine().h2d_bytes += (long long)b; }
inline void count_d2h(size_t b) { engine().d2h_bytes += (long long)b; }
// Kernel launches are counted process-wide and per thread; a thread that
// captures a CUDA graph measures the graph's launches on its own counter,
// which launches of other threads in the meantime leave alone.
extern thread_local long long tls_launches;
inline void count_launch(int n = 1)
{
    engine().launches += n;
    tls_launches += n;
}

// cudaMemcpyAsync that also counts the bytes it moves between host and device
inline cudaError_t counted_memcpy(void *dst, const void *src, size_t n, cudaMemcpyKind kind, cudaStream_t st)
{
    if (kind == cudaMemcpyHostToDevice) count_h2d(n);
    else if (kind == cudaMemcpyDeviceToHost) count_d2h(n);
    return cudaMemcpyAsync(dst, src, n, kind, st);
}

// ---- staged copies between pageable host memory and the device -------------
// A pageable cudaMemcpy moves through the driver's own small staging at a
// fraction of the link's speed.  These copy a list of spans through the
// context's pinned stage instead, in chunks of STAGE_CHUNK bytes: host
// threads fill one half of the stage while the copy engine drains the other.
// Both return once every copy has completed (the stage is free again).
struct HostSpan {
    void *host;
    void *dev;
    size_t bytes;
};
constexpr size_t STAGE_CHUNK = (size_t)32 << 20;
// Host copy with non-temporal stores: the destination lines are written
// without being read first, which takes a third of the memory traffic off a
// large copy between pageable memory and a pinned stage.
void copy_nt(void *dst, const void *src, size_t n);
Status staged_upload(const HostSpan *spans, int n, const Ctx &ctx);
Status staged_download(const HostSpan *spans, int n, const Ctx &ctx);
// the same upload through a given stage, on a given stream (the caller's
// thread must have the stream's device current)
Status staged_upload_via(const HostSpan *spans, int n, Pinned *stage, cudaStream_t st);

// ---- device utilities (scan.cu) -------------------------------------------
// out[i] = sum_{j<i} in[i] for i in [0, n], out[n] = total.  `tmp` must hold
// scan_tmp_elems(n) int64 values.
size_t scan_tmp_elems(long long n);
Status exclusive_scan_i32(const int *in, long long *out, long long n, long long *tmp, cudaStream_t st);
Status exclusive_scan_i64(const long long *in, long long *out, long long n, long long *tmp, cudaStream_t st);

// ---- single-graph fit (fit_graph.cu) --------------------------------------
struct FitStats {
    long long T = 0;            // common-neighbour terms per sweep
    int sweeps = 0;             // sweeps executed
    double setup_ms = 0, iterate_ms = 0;
    // host time of the fit's phases: upload, validation, common-neighbour
    // tables and bins, renumbering and sweep set-up, results download
    double phase_ms[5] = {};
    long long vbin_items[8] = {}, vbin_terms[8] = {}, ebin_items[8] = {}, ebin_terms[8] = {};
};
Status fit_graph(p_dress_graph_t g, int max_iterations, double epsilon,
                 int *iterations, double *delta, FitStats *stats, const Ctx &ctx);
// The same fit in one launch for graphs whose state fits one SM (fit_small.cu);
// `used` is false, and nothing is done, for the others.
Status fit_small(p_dress_graph_t g, int max_iterations, double epsilon, int *iterations, double *delta,
                 FitStats *stats, const Ctx &ctx, bool &used);

// ---- Delta/Nabla requests (delta_nabla.cpp) ---------------------------------
// edge_sweeps (nullable, n entries): live edges x sweeps summed over each
// request's fits.
Status hist_batch_core(dressx_hist_request_t *reqs, int n, bool per_fit, const Ctx &ctx,
                       int64_t *edge_sweeps = nullptr);

}  // namespace dress
