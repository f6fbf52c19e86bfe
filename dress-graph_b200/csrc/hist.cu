// hist.cu -- exact (value, count) histograms of many value segments.
//
// Reference: libdress/src/dress_histogram.c:40-155 -- a hash map keyed on the
// exact double (equality by ==) flattened to [bits, count] pairs sorted
// ascending by value.  Here every request's converged edge values sit in one
// contiguous segment of a device buffer; all segments are sorted at once by a
// segmented LSD radix sort on the order-preserving 64-bit image of the double
// (8-bit digits, stable in-tile ranking), then run-length encoded.  A run is
// one bit pattern, as the reference's map keys values by their bits (its
// hash reads the pattern) and merges them by ==: the only ==-equal values it
// can keep apart, +0 and -0, hash to different slots and merge only when
// one's probe run reaches the other; here they are two entries, -0 first.
// Every NaN is a run of its own (never == itself), as in the map.  A pass in
// which every segment has a single digit value moves nothing and is skipped.
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <thread>
#include <condition_variable>
#include <vector>

#include "engine.h"
#include "hist.h"
#include "host_par.h"

namespace dress {
namespace {

constexpr int HT = 512;                 // threads per tile block
constexpr int HI = 16;                  // keys per thread per tile
constexpr int TILE = HT * HI;           // 8192 keys per tile
constexpr int RADIX = 256;

__device__ __forceinline__ unsigned long long to_ordered(unsigned long long b)
{
    return (b >> 63) ? ~b : (b | 0x8000000000000000ULL);
}
__device__ __forceinline__ unsigned long long from_ordered(unsigned long long k)
{
    return (k >> 63) ? (k & 0x7fffffffffffffffULL) : ~k;
}

__device__ __forceinline__ unsigned lanemask_lt_h()
{
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

struct Tile {
    long long begin, end;   // key range
    int seg;
};

__global__ void k_to_ordered(long long n, unsigned long long *k)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        k[i] = to_ordered(k[i]);
}

// per-tile digit counts
__global__ void __launch_bounds__(HT) k_tile_hist(const Tile *tiles, const unsigned long long *keys,
                                                  int shift, int *counts)
{
    __shared__ int c[RADIX];
    Tile t = tiles[blockIdx.x];
    for (int d = threadIdx.x; d < RADIX; d += HT) c[d] = 0;
    __syncthreads();
    for (long long i = t.begin + threadIdx.x; i < t.end; i += HT)
        atomicAdd(&c[(keys[i] >> shift) & 0xff], 1);
    __syncthreads();
    for (int d = threadIdx.x; d < RADIX; d += HT) counts[(long long)blockIdx.x * RADIX + d] = c[d];
}

// per segment: scatter offsets of every (tile, digit); flags a pass that moves keys
__global__ void __launch_bounds__(RADIX) k_seg_offsets(const long long *seg_begin, const int *seg_tile0,
                                                       const int *counts, long long *offs, int *moves)
{
    __shared__ long long base[RADIX];
    __shared__ int nonzero;
    int s = blockIdx.x, d = threadIdx.x;
    int t0 = seg_tile0[s], t1 = seg_tile0[s + 1];
    long long tot = 0;
    for (int t = t0; t < t1; ++t) tot += counts[(long long)t * RADIX + d];
    if (d == 0) nonzero = 0;
    base[d] = tot;
    __syncthreads();
    if (tot > 0) atomicAdd(&nonzero, 1);
    if (d == 0) {
        long long run = seg_begin[s];
        for (int k = 0; k < RADIX; ++k) {
            long long c = base[k];
            base[k] = run;
            run += c;
        }
    }
    __syncthreads();
    if (nonzero > 1 && d == 0) *moves = 1;
    long long run = base[d];
    for (int t = t0; t < t1; ++t) {
        offs[(long long)t * RADIX + d] = run;
        run += counts[(long long)t * RADIX + d];
    }
}

// The same offsets for one long segment, in parallel: per chunk of
// OFF_CHUNK tiles the digit sums (k_chunk_sums), then the digit bases and
// every chunk's base per digit (k_chunk_bases, one block over the chunks),
// then each chunk's tiles (k_chunk_fill).  k_seg_offsets walks every tile of
// its segment with one block, which makes a segment of 10^8 keys (12K tiles)
// cost milliseconds per pass.
constexpr int OFF_CHUNK = 64;

__global__ void __launch_bounds__(RADIX) k_chunk_sums(int nt, const int *counts, long long *csum)
{
    const int c = blockIdx.x, d = threadIdx.x;
    const int t1 = min(nt, (c + 1) * OFF_CHUNK);
    long long sum = 0;
    for (int t = c * OFF_CHUNK; t < t1; ++t) sum += counts[(long long)t * RADIX + d];
    csum[(long long)c * RADIX + d] = sum;
}

__global__ void __launch_bounds__(RADIX) k_chunk_bases(int nch, const long long *seg_begin, long long *csum,
                                                       int *moves)
{
    __shared__ long long base[RADIX];
    __shared__ int nonzero;
    const int d = threadIdx.x;
    long long tot = 0;
    for (int c = 0; c < nch; ++c) tot += csum[(long long)c * RADIX + d];
    if (d == 0) nonzero = 0;
    base[d] = tot;
    __syncthreads();
    if (tot > 0) atomicAdd(&nonzero, 1);
    if (d == 0) {
        long long run = seg_begin[0];
        for (int k = 0; k < RADIX; ++k) {
            const long long c = base[k];
            base[k] = run;
            run += c;
        }
    }
    __syncthreads();
    if (nonzero > 1 && d == 0) *moves = 1;
    long long run = base[d];
    for (int c = 0; c < nch; ++c) {
        const long long v = csum[(long long)c * RADIX + d];
        csum[(long long)c * RADIX + d] = run;
        run += v;
    }
}

__global__ void __launch_bounds__(RADIX) k_chunk_fill(int nt, const int *counts, const long long *cbase,
                                                      long long *offs)
{
    const int c = blockIdx.x, d = threadIdx.x;
    const int t1 = min(nt, (c + 1) * OFF_CHUNK);
    long long run = cbase[(long long)c * RADIX + d];
    for (int t = c * OFF_CHUNK; t < t1; ++t) {
        offs[(long long)t * RADIX + d] = run;
        run += counts[(long long)t * RADIX + d];
    }
}

// stable scatter of one tile: rounds of HT consecutive keys, each key ranked
// by (its rank among equal digits in its warp) + (same digit in earlier warps
// of the round) + (same digit in earlier rounds of the tile)
__global__ void __launch_bounds__(HT) k_tile_scatter(const Tile *tiles, const unsigned long long *src,
                                                     unsigned long long *dst, int shift,
                                                     const long long *offs, const unsigned *psrc, unsigned *pdst)
{
    constexpr int W = HT / 32;
    __shared__ int wcnt[W][RADIX];
    __shared__ int rtot[RADIX];
    __shared__ long long dbase[RADIX];
    Tile t = tiles[blockIdx.x];
    int wid = threadIdx.x >> 5;
    for (int d = threadIdx.x; d < RADIX; d += HT) dbase[d] = offs[(long long)blockIdx.x * RADIX + d];
    for (long long r0 = t.begin; r0 < t.end; r0 += HT) {
        for (int q = threadIdx.x; q < W * RADIX; q += HT) (&wcnt[0][0])[q] = 0;
        __syncthreads();
        long long i = r0 + threadIdx.x;
        bool valid = i < t.end;
        unsigned long long key = valid ? src[i] : 0ULL;
        int dg = valid ? (int)((key >> shift) & 0xff) : RADIX;      // RADIX: no key
        unsigned peers = __match_any_sync(0xffffffffu, dg);
        int rank = __popc(peers & lanemask_lt_h());
        if (valid && rank == 0) wcnt[wid][dg] = __popc(peers);
        __syncthreads();
        for (int d = threadIdx.x; d < RADIX; d += HT) {
            int run = 0;
            for (int w = 0; w < W; ++w) {
                int c = wcnt[w][d];
                wcnt[w][d] = run;
                run += c;
            }
            rtot[d] = run;
        }
        __syncthreads();
        if (valid) {
            const long long pos = dbase[dg] + wcnt[wid][dg] + rank;
            dst[pos] = key;
            if (pdst) pdst[pos] = psrc[i];          // payload moves with its key
        }
        __syncthreads();
        for (int d = threadIdx.x; d < RADIX; d += HT) dbase[d] += rtot[d];
        __syncthreads();
    }
}

// run heads per tile: segments start a run, a new bit pattern starts one,
// and so does every NaN
__device__ __forceinline__ bool is_head(const unsigned long long *k, long long i, long long seg_begin)
{
    if (i == seg_begin || k[i] != k[i - 1]) return true;
    const double a = __longlong_as_double((long long)from_ordered(k[i]));
    return a != a;
}

__global__ void __launch_bounds__(HT) k_tile_heads(const Tile *tiles, const long long *seg_begin,
                                                   const unsigned long long *keys, long long *tile_heads)
{
    __shared__ int cnt;
    Tile t = tiles[blockIdx.x];
    if (threadIdx.x == 0) cnt = 0;
    __syncthreads();
    long long sb = seg_begin[t.seg];
    int c = 0;
    for (long long i = t.begin + threadIdx.x; i < t.end; i += HT) c += is_head(keys, i, sb);
    atomicAdd(&cnt, c);
    __syncthreads();
    if (threadIdx.x == 0) tile_heads[blockIdx.x] = cnt;
}

// write (value bits, start) of every run in order; counts follow from starts
__global__ void __launch_bounds__(HT) k_tile_runs(const Tile *tiles, const long long *seg_begin,
                                                  const unsigned long long *keys, const long long *tile_base,
                                                  long long *run_start, unsigned long long *run_bits,
                                                  int *run_seg)
{
    __shared__ int wsum[HT / 32];
    __shared__ long long carry;
    Tile t = tiles[blockIdx.x];
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    long long sb = seg_begin[t.seg];
    if (threadIdx.x == 0) carry = tile_base[blockIdx.x];
    __syncthreads();
    for (long long r0 = t.begin; r0 < t.end; r0 += HT) {
        long long i = r0 + threadIdx.x;
        bool h = i < t.end && is_head(keys, i, sb);
        unsigned b = __ballot_sync(0xffffffffu, h);
        if (lane == 0) wsum[wid] = __popc(b);
        __syncthreads();
        int before = 0, total = 0;
        for (int w = 0; w < HT / 32; ++w) {
            int c = wsum[w];
            if (w < wid) before += c;
            total += c;
        }
        if (h) {
            long long r = carry + before + __popc(b & lanemask_lt_h());
            run_start[r] = i;
            run_bits[r] = from_ordered(keys[i]);
            run_seg[r] = t.seg;
        }
        __syncthreads();
        if (threadIdx.x == 0) carry += total;
        __syncthreads();
    }
}

__global__ void k_run_pairs(long long R, const long long *run_start, const unsigned long long *run_bits,
                            const int *run_seg, const long long *seg_end, long long *pairs)
{
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < R;
         r += (long long)gridDim.x * blockDim.x) {
        int s = run_seg[r];
        long long end = (r + 1 < R && run_seg[r + 1] == s) ? run_start[r + 1] : seg_end[s];
        pairs[2 * r] = (long long)run_bits[r];
        pairs[2 * r + 1] = end - run_start[r];
    }
}

// Tiles of the segments, uploaded, and the keys sorted (order-preserving
// image) within every segment; `out` is the buffer holding the result.
struct SortPlan {
    DevBuf<Tile> tiles;
    DevBuf<long long> seg_begin, seg_end;
    int nt = 0, nseg = 0;
    unsigned long long *out = nullptr;
    unsigned *pout = nullptr;
};

// ordered: keys are raw double bits, sorted by value through their
// order-preserving image (left in place); otherwise they are unsigned
// integers.  vals/valt (nullable): a 32-bit payload moved with the keys.
// key_bits < 64: the keys are below 2^key_bits, so only the passes over those
// bits run, each unconditionally (no host check of whether it moves keys).
Status sort_segments(unsigned long long *keys, unsigned long long *alt, const std::vector<long long> &begin,
                     const std::vector<long long> &len, SortPlan &sp, cudaStream_t st, int sms,
                     bool ordered = true, unsigned *vals = nullptr, unsigned *valt = nullptr, int key_bits = 64)
{
    const int nseg = (int)begin.size();
    sp.nseg = nseg;
    sp.out = keys;
    sp.pout = vals;
    std::vector<Tile> tiles;
    std::vector<int> seg_tile0((size_t)nseg + 1, 0);
    std::vector<long long> seg_end((size_t)nseg);
    long long total = 0, lo = -1, hi = 0;
    for (int s = 0; s < nseg; ++s) {
        seg_tile0[(size_t)s] = (int)tiles.size();
        seg_end[(size_t)s] = begin[(size_t)s] + len[(size_t)s];
        for (long long b = begin[(size_t)s]; b < seg_end[(size_t)s]; b += TILE)
            tiles.push_back({b, b + TILE < seg_end[(size_t)s] ? b + TILE : seg_end[(size_t)s], s});
        total += len[(size_t)s];
        if (len[(size_t)s] > 0) {
            if (lo < 0 || begin[(size_t)s] < lo) lo = begin[(size_t)s];
            if (seg_end[(size_t)s] > hi) hi = seg_end[(size_t)s];
        }
    }
    seg_tile0[(size_t)nseg] = (int)tiles.size();
    sp.nt = (int)tiles.size();
    if (total == 0) return Status::Ok();
    const int nt = sp.nt;

    DevBuf<int> d_seg_tile0, d_counts, d_moves;
    DevBuf<long long> d_offs;
    DRESS_TRY(sp.tiles.alloc((size_t)nt, st));
    DRESS_TRY(d_seg_tile0.alloc((size_t)nseg + 1, st));
    DRESS_TRY(sp.seg_begin.alloc((size_t)nseg, st));
    DRESS_TRY(sp.seg_end.alloc((size_t)nseg, st));
    DRESS_TRY(d_counts.alloc((size_t)nt * RADIX, st));
    DRESS_TRY(d_offs.alloc((size_t)nt * RADIX, st));
    DRESS_TRY(d_moves.alloc(1, st));
    DRESS_CUDA_TRY(counted_memcpy(sp.tiles.get(), tiles.data(), (size_t)nt * sizeof(Tile), cudaMemcpyHostToDevice, st));
    DRESS_CUDA_TRY(counted_memcpy(d_seg_tile0.get(), seg_tile0.data(), ((size_t)nseg + 1) * sizeof(int),
                                   cudaMemcpyHostToDevice, st));
    DRESS_CUDA_TRY(counted_memcpy(sp.seg_begin.get(), begin.data(), (size_t)nseg * sizeof(long long),
                                   cudaMemcpyHostToDevice, st));
    DRESS_CUDA_TRY(counted_memcpy(sp.seg_end.get(), seg_end.data(), (size_t)nseg * sizeof(long long),
                                   cudaMemcpyHostToDevice, st));

    // order-preserving image of the doubles over the used span
    if (ordered)
        count_launch(), k_to_ordered<<<(unsigned)((hi - lo + 255) / 256 < 64 * sms ? (hi - lo + 255) / 256 : 64 * sms), 256, 0, st>>>(
            hi - lo, keys + lo);
    unsigned long long *a = keys, *b = alt;
    unsigned *pa = vals, *pb = valt;
    const bool chunked = nseg == 1 && nt >= 4 * OFF_CHUNK;
    const int nch = (nt + OFF_CHUNK - 1) / OFF_CHUNK;
    DevBuf<long long> d_csum;
    if (chunked) DRESS_TRY(d_csum.alloc((size_t)nch * RADIX, st));
    const bool check = key_bits >= 64;
    const int passes = check ? 8 : std::max(1, (key_bits + 7) / 8);
    for (int pass = 0; pass < passes; ++pass) {
        int shift = 8 * pass;
        count_launch(), k_tile_hist<<<nt, HT, 0, st>>>(sp.tiles.get(), a, shift, d_counts.get());
        if (check) DRESS_CUDA_TRY(cudaMemsetAsync(d_moves.get(), 0, sizeof(int), st));
        if (chunked) {
            count_launch(), k_chunk_sums<<<nch, RADIX, 0, st>>>(nt, d_counts.get(), d_csum.get());
            count_launch(), k_chunk_bases<<<1, RADIX, 0, st>>>(nch, sp.seg_begin.get(), d_csum.get(), d_moves.get());
            count_launch(), k_chunk_fill<<<nch, RADIX, 0, st>>>(nt, d_counts.get(), d_csum.get(), d_offs.get());
        } else {
            count_launch(), k_seg_offsets<<<nseg, RADIX, 0, st>>>(sp.seg_begin.get(), d_seg_tile0.get(),
                                                                  d_counts.get(), d_offs.get(), d_moves.get());
        }
        if (check) {
            int moves = 0;
            DRESS_CUDA_TRY(counted_memcpy(&moves, d_moves.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
            DRESS_CUDA_TRY(cudaStreamSynchronize(st));
            if (!moves) continue;
        }
        count_launch(), k_tile_scatter<<<nt, HT, 0, st>>>(sp.tiles.get(), a, b, shift, d_offs.get(), pa, pb);
        unsigned long long *t = a;
        a = b;
        b = t;
        unsigned *tp = pa;
        pa = pb;
        pb = tp;
    }
    DRESS_CUDA_TRY(cudaGetLastError());
    sp.out = a;
    sp.pout = pa;
    return Status::Ok();
}

}  // namespace

Status segmented_sort(unsigned long long *keys, unsigned long long *alt, const std::vector<long long> &begin,
                      const std::vector<long long> &len, unsigned long long **sorted, cudaStream_t st, int sms)
{
    SortPlan sp;
    DRESS_TRY(sort_segments(keys, alt, begin, len, sp, st, sms));
    *sorted = sp.out;
    return Status::Ok();
}

Status sort_pairs(unsigned long long *keys, unsigned long long *alt, unsigned *vals, unsigned *valt, long long n,
                  unsigned long long **sorted_keys, unsigned **sorted_vals, cudaStream_t st, int sms, int key_bits)
{
    SortPlan sp;
    DRESS_TRY(sort_segments(keys, alt, std::vector<long long>{0}, std::vector<long long>{n}, sp, st, sms, false,
                            vals, valt, key_bits));
    *sorted_keys = sp.out;
    *sorted_vals = sp.pout;
    return Status::Ok();
}

Status histogram_device(unsigned long long *keys, unsigned long long *alt, const std::vector<long long> &begin,
                        const std::vector<long long> &len, HistResult &res, cudaStream_t st, int sms)
{
    const int nseg = (int)begin.size();
    res.nseg = nseg;
    res.R = 0;
    long long total = 0;
    for (long long l : len) total += l;
    if (total == 0) return Status::Ok();
    SortPlan sp;
    DRESS_TRY(sort_segments(keys, alt, begin, len, sp, st, sms));
    const int nt = sp.nt;
    unsigned long long *a = sp.out;
    DevBuf<long long> d_tile_heads, d_tile_base, d_scan_tmp, d_run_start;
    DevBuf<unsigned long long> d_run_bits;

    // run-length encode
    DRESS_TRY(d_tile_heads.alloc((size_t)nt, st));
    DRESS_TRY(d_tile_base.alloc((size_t)nt + 1, st));
    DRESS_TRY(d_scan_tmp.alloc(scan_tmp_elems(nt), st));
    count_launch(), k_tile_heads<<<nt, HT, 0, st>>>(sp.tiles.get(), sp.seg_begin.get(), a, d_tile_heads.get());
    DRESS_TRY(exclusive_scan_i64(d_tile_heads.get(), d_tile_base.get(), nt, d_scan_tmp.get(), st));
    long long R = 0;
    DRESS_CUDA_TRY(counted_memcpy(&R, d_tile_base.get() + nt, sizeof(R), cudaMemcpyDeviceToHost, st));
    DRESS_CUDA_TRY(cudaStreamSynchronize(st));
    DRESS_TRY(d_run_start.alloc((size_t)R, st));
    DRESS_TRY(d_run_bits.alloc((size_t)R, st));
    DRESS_TRY(res.run_seg.alloc((size_t)R, st));
    DRESS_TRY(res.pairs.alloc(2 * (size_t)R, st));
    count_launch(), k_tile_runs<<<nt, HT, 0, st>>>(sp.tiles.get(), sp.seg_begin.get(), a, d_tile_base.get(), d_run_start.get(),
                                   d_run_bits.get(), res.run_seg.get());
    count_launch(), k_run_pairs<<<(unsigned)((R + 255) / 256 < 64 * sms ? (R + 255) / 256 : 64 * sms), 256, 0, st>>>(
        R, d_run_start.get(), d_run_bits.get(), res.run_seg.get(), sp.seg_end.get(), res.pairs.get());
    DRESS_CUDA_TRY(cudaGetLastError());
    res.R = R;
    return Status::Ok();
}

// end (one past the last run) of every segment that has runs
__global__ void k_seg_ends(long long R, const int *run_seg, long long *seg_end)
{
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < R;
         r += (long long)gridDim.x * blockDim.x)
        if (r + 1 == R || run_seg[r + 1] != run_seg[r]) seg_end[run_seg[r]] = r + 1;
}

Status histogram_fetch(HistResult &res, std::vector<int64_t *> &outs, std::vector<long long> &lens, Pinned *stage,
                       cudaStream_t st, int sms, std::vector<int64_t *> *pre, const std::vector<long long> *cap,
                       int max_threads)
{
    const int nseg = res.nseg;
    outs.assign((size_t)nseg, nullptr);
    lens.assign((size_t)nseg, 0);
    const long long R = res.R;
    if (R == 0) return Status::Ok();
    DevBuf<long long> d_end;
    DRESS_TRY(d_end.alloc((size_t)nseg, st));
    DRESS_CUDA_TRY(cudaMemsetAsync(d_end.get(), 0, (size_t)nseg * sizeof(long long), st));
    count_launch(), k_seg_ends<<<(unsigned)((R + 255) / 256 < 16 * sms ? (R + 255) / 256 : 16 * sms), 256, 0, st>>>(
        R, res.run_seg.get(), d_end.get());
    std::vector<long long> end((size_t)nseg);
    DRESS_CUDA_TRY(counted_memcpy(end.data(), d_end.get(), (size_t)nseg * sizeof(long long), cudaMemcpyDeviceToHost, st));
    DRESS_CUDA_TRY(cudaStreamSynchronize(st));
    // runs are grouped by segment in segment order: a segment starts where the
    // last non-empty one before it ended
    std::vector<long long> first((size_t)nseg, 0);
    long long prev = 0;
    for (int sg = 0; sg < nseg; ++sg) {
        if (end[(size_t)sg] > 0) {
            first[(size_t)sg] = prev;
            lens[(size_t)sg] = 2 * (end[(size_t)sg] - prev);
            prev = end[(size_t)sg];
        }
    }
    const size_t bytes = 2 * (size_t)R * sizeof(long long);
    long long *host = nullptr;
    std::vector<long long> pageable;
    const bool pinned = stage && stage->reserve(bytes).ok();
    if (pinned) {
        host = (long long *)stage->ptr();
    } else {
        pageable.resize(2 * (size_t)R);
        host = pageable.data();
    }
    // The output, runs [0, R) in segment order, is cut into one part per host
    // thread, balanced by bytes; each part is its own download.  A thread
    // allocates the arrays of the segments that start in its part, and after
    // a barrier (a segment may reach into later parts) maps the pages of its
    // part's share of the arrays while the downloads stream in -- the page
    // faults of fresh memory cost more than the copy -- then copies its
    // share once its part landed.  A final barrier precedes the trimming of
    // given arrays to their length.
    const int nthr = pinned && bytes > (64u << 20) ? std::min(max_threads, host_threads((long long)(bytes >> 23))) : 1;
    const int parts = std::max(1, nthr);
    std::vector<long long> pcut((size_t)parts + 1);
    for (int t = 0; t <= parts; ++t) pcut[(size_t)t] = R * t / parts;
    std::vector<cudaEvent_t> ev((size_t)parts, nullptr);
    Status err;
    for (int t = 0; t < parts && err.ok(); ++t) {
        const long long r0 = pcut[(size_t)t], r1 = pcut[(size_t)t + 1];
        if (r1 <= r0) continue;
        if (cudaEventCreateWithFlags(&ev[(size_t)t], cudaEventDisableTiming | cudaEventBlockingSync) != cudaSuccess) {
            ev[(size_t)t] = nullptr;
            err = Status::Err(DRESSX_ECUDA, "event creation failed");
            break;
        }
        cudaError_t e = counted_memcpy(host + 2 * r0, res.pairs.get() + 2 * r0, 2 * (size_t)(r1 - r0) * sizeof(long long),
                                       cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaEventRecord(ev[(size_t)t], st);
        if (e != cudaSuccess) err = Status::Err(DRESSX_ECUDA, std::string("histogram download: ") + cudaGetErrorString(e));
    }
    // segments in part order: the first segment whose runs reach into each part
    std::vector<int> seg0((size_t)parts + 1, nseg);
    {
        int sg = 0;
        for (int t = 0; t < parts; ++t) {
            while (sg < nseg && (lens[(size_t)sg] == 0 || first[(size_t)sg] + lens[(size_t)sg] / 2 <= pcut[(size_t)t]))
                ++sg;
            seg0[(size_t)t] = sg;
        }
    }
    std::vector<char> given((size_t)nseg, 0);    // segments that took a given array
    std::atomic<bool> nomem{false};
    std::mutex mu;
    std::condition_variable cv;
    int ready = 0;                               // parts landed; -1 once the downloads failed
    int arrived[2] = {0, 0};                     // barrier counts
    auto barrier = [&](int b) {
        std::unique_lock<std::mutex> lk(mu);
        if (++arrived[b] == parts) cv.notify_all();
        else cv.wait(lk, [&] { return arrived[b] == parts; });
    };
    auto part_work = [&](int t) {
        const long long p0 = pcut[(size_t)t], p1 = pcut[(size_t)t + 1];
        // the segments starting in this part
        for (int sg = seg0[(size_t)t]; sg < nseg && first[(size_t)sg] < p1; ++sg) {
            const size_t n = (size_t)lens[(size_t)sg] * sizeof(int64_t);
            if (!n || first[(size_t)sg] < p0) continue;
            if (pre && (*pre)[(size_t)sg] && lens[(size_t)sg] <= (*cap)[(size_t)sg]) {
                outs[(size_t)sg] = (*pre)[(size_t)sg];
                (*pre)[(size_t)sg] = nullptr;
                given[(size_t)sg] = 1;
                continue;
            }
            outs[(size_t)sg] = (int64_t *)std::malloc(n);
            if (!outs[(size_t)sg]) nomem = true;
        }
        barrier(0);
        // this part's share of segment sg: runs [a, b)
        auto share = [&](int sg, long long &a, long long &b) {
            a = std::max(p0, first[(size_t)sg]);
            b = std::min(p1, first[(size_t)sg] + lens[(size_t)sg] / 2);
        };
        if (parts > 1)
            for (int sg = seg0[(size_t)t]; sg < nseg && first[(size_t)sg] < p1; ++sg) {
                long long a, b;
                share(sg, a, b);
                char *o = (char *)outs[(size_t)sg];
                if (b <= a || !o || given[(size_t)sg]) continue;
                const size_t lo_b = (size_t)(a - first[(size_t)sg]) * 16, hi_b = (size_t)(b - first[(size_t)sg]) * 16;
                for (size_t x = lo_b; x < hi_b; x += 4096) ((volatile char *)o)[x] = 0;
            }
        bool ok;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv.wait(lk, [&] { return ready < 0 || ready > t; });
            ok = ready > t;
        }
        if (ok)
            for (int sg = seg0[(size_t)t]; sg < nseg && first[(size_t)sg] < p1; ++sg) {
                long long a, b;
                share(sg, a, b);
                int64_t *o = outs[(size_t)sg];
                if (b <= a || !o) continue;
                copy_nt(o + 2 * (a - first[(size_t)sg]), host + 2 * a, (size_t)(b - a) * 16);
            }
        barrier(1);
        // trim the given arrays of the segments starting here (shrinking keeps the data)
        for (int sg = seg0[(size_t)t]; sg < nseg && first[(size_t)sg] < p1; ++sg)
            if (given[(size_t)sg] && first[(size_t)sg] >= p0 && lens[(size_t)sg] < (*cap)[(size_t)sg]) {
                void *r2 = std::realloc(outs[(size_t)sg], (size_t)lens[(size_t)sg] * sizeof(int64_t));
                if (r2) outs[(size_t)sg] = (int64_t *)r2;
            }
    };
    std::vector<std::thread> th;
    if (parts > 1)
        for (int t = 0; t < parts; ++t) th.emplace_back(part_work, t);
    // this thread waits for the downloads in order and releases the parts
    for (int t = 0; t < parts && err.ok(); ++t) {
        if (ev[(size_t)t] && cudaEventSynchronize(ev[(size_t)t]) != cudaSuccess) {
            err = Status::Err(DRESSX_ECUDA, "histogram download failed");
        } else {
            std::lock_guard<std::mutex> lk(mu);
            ready = t + 1;
            cv.notify_all();
        }
    }
    if (!err.ok()) {
        std::lock_guard<std::mutex> lk(mu);
        ready = -1;
        cv.notify_all();
    }
    if (parts == 1) part_work(0);
    for (auto &t : th) t.join();
    for (cudaEvent_t e : ev)
        if (e) cudaEventDestroy(e);
    if (err.ok() && nomem) err = Status::Err(DRESSX_ENOMEM, "host allocation of the histograms failed");
    if (!err.ok()) {
        for (auto &o : outs) std::free(o);
        outs.assign((size_t)nseg, nullptr);
    }
    return err;
}

Status histogram_download(HistResult &res, std::vector<std::vector<long long>> &out, cudaStream_t st)
{
    out.assign((size_t)res.nseg, std::vector<long long>());
    const long long R = res.R;
    if (R == 0) return Status::Ok();
    std::vector<long long> pairs(2 * (size_t)R);
    std::vector<int> rseg((size_t)R);
    DRESS_CUDA_TRY(counted_memcpy(pairs.data(), res.pairs.get(), 2 * (size_t)R * sizeof(long long),
                                   cudaMemcpyDeviceToHost, st));
    DRESS_CUDA_TRY(counted_memcpy(rseg.data(), res.run_seg.get(), (size_t)R * sizeof(int), cudaMemcpyDeviceToHost, st));
    DRESS_CUDA_TRY(cudaStreamSynchronize(st));
    // runs come out grouped by segment, in segment order
    long long r = 0;
    while (r < R) {
        int sgm = rseg[(size_t)r];
        long long e = r;
        while (e < R && rseg[(size_t)e] == sgm) ++e;
        out[(size_t)sgm].assign(pairs.begin() + 2 * r, pairs.begin() + 2 * e);
        r = e;
    }
    return Status::Ok();
}

Status histogram_segments(unsigned long long *keys, unsigned long long *alt, const std::vector<long long> &begin,
                          const std::vector<long long> &len, std::vector<std::vector<long long>> &out,
                          cudaStream_t st, int sms)
{
    HistResult res;
    DRESS_TRY(histogram_device(keys, alt, begin, len, res, st, sms));
    return histogram_download(res, out, st);
}

}  // namespace dress

// ---------------------------------------------------------------------------
// Histogram without any allocation (dressx_histogram_noalloc)
//
// Some callers cannot allocate device memory at the moment they need a
// histogram: code running while a CUDA graph is being captured, frameworks
// whose caching allocator owns all device memory, or real-time loops that
// forbid allocation after start-up.  For them the pipeline above runs on one
// segment of at most NOALLOC_MAX values with every scratch buffer carved out
// of the file-scope array below.  Every GPU that loads this library holds the
// array (about 16.5 MiB) until the process exits.  The call only enqueues work
// on the caller's stream (no host synchronisation, all eight digit passes
// always run), so results are ready when the stream reaches that point.  All
// calls share the one array: calls whose work overlaps on the GPU race.
// ---------------------------------------------------------------------------
namespace dress {
namespace {

constexpr long long NOALLOC_MAX = DRESSX_NOALLOC_MAX_VALUES;
constexpr int NA_TILES = (int)(NOALLOC_MAX / TILE);
static_assert(NOALLOC_MAX % TILE == 0, "whole tiles");

// byte offsets of the carved buffers
constexpr long long NA_A = 0;                                       // u64 keys, sorted here
constexpr long long NA_B = NA_A + 8 * NOALLOC_MAX;                  // u64 ping-pong / run starts
constexpr long long NA_OFFS = NA_B + 8 * NOALLOC_MAX;               // i64 [tiles][256]
constexpr long long NA_COUNTS = NA_OFFS + 8LL * NA_TILES * RADIX;   // i32 [tiles][256]
constexpr long long NA_TILESB = NA_COUNTS + 4LL * NA_TILES * RADIX; // Tile [tiles]
constexpr long long NA_HEADS = NA_TILESB + 32LL * NA_TILES;         // i64 [tiles]
constexpr long long NA_BASE = NA_HEADS + 8LL * NA_TILES;            // i64 [tiles+1]
constexpr long long NA_SEG = NA_BASE + 8LL * (NA_TILES + 8);                          // i64 begin, i64 end, i32 tile0[2], i32 moves
constexpr long long NA_BYTES = NA_SEG + 64;
static_assert(sizeof(Tile) <= 32, "tile descriptor slot");

static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

// single segment [0, n): tile descriptors and segment bounds
__global__ void k_na_setup(long long n, int nt, Tile *tiles, long long *seg_begin, long long *seg_end,
                           int *seg_tile0)
{
    for (int t = threadIdx.x; t < nt; t += blockDim.x) {
        long long b = (long long)t * TILE;
        tiles[t].begin = b;
        tiles[t].end = b + TILE < n ? b + TILE : n;
        tiles[t].seg = 0;
    }
    if (threadIdx.x == 0) {
        seg_begin[0] = 0;
        seg_end[0] = n;
        seg_tile0[0] = 0;
        seg_tile0[1] = nt;
    }
}

__global__ void k_na_load(long long n, const double *in, unsigned long long *keys)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        keys[i] = to_ordered((unsigned long long)__double_as_longlong(in[i]));
}

// run starts into `starts`, value bits into pairs[2r]
__global__ void __launch_bounds__(HT) k_na_runs(const Tile *tiles, const unsigned long long *keys,
                                                const long long *tile_base, long long *starts, long long *pairs)
{
    __shared__ int wsum[HT / 32];
    __shared__ long long carry;
    Tile t = tiles[blockIdx.x];
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (threadIdx.x == 0) carry = tile_base[blockIdx.x];
    __syncthreads();
    for (long long r0 = t.begin; r0 < t.end; r0 += HT) {
        long long i = r0 + threadIdx.x;
        bool h = i < t.end && is_head(keys, i, 0);
        unsigned b = __ballot_sync(0xffffffffu, h);
        if (lane == 0) wsum[wid] = __popc(b);
        __syncthreads();
        int before = 0, total = 0;
        for (int w = 0; w < HT / 32; ++w) {
            int c = wsum[w];
            if (w < wid) before += c;
            total += c;
        }
        if (h) {
            long long r = carry + before + __popc(b & lanemask_lt_h());
            starts[r] = i;
            pairs[2 * r] = (long long)from_ordered(keys[i]);
        }
        __syncthreads();
        if (threadIdx.x == 0) carry += total;
        __syncthreads();
    }
}

// exclusive prefix of the per-tile head counts (nt <= NA_TILES values)
__global__ void k_na_scan(const long long *heads, int nt, long long *tile_base)
{
    if (threadIdx.x != 0) return;
    long long run = 0;
    for (int t = 0; t < nt; ++t) {
        tile_base[t] = run;
        run += heads[t];
    }
    tile_base[nt] = run;
}

// counts from consecutive run starts; the run total sits at tile_base[nt]
__global__ void k_na_counts(long long n, int nt, const long long *tile_base, const long long *starts,
                            long long *pairs, long long *num_runs)
{
    const long long R = tile_base[nt];
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < R;
         r += (long long)gridDim.x * blockDim.x) {
        long long end = r + 1 < R ? starts[r + 1] : n;
        pairs[2 * r + 1] = end - starts[r];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *num_runs = R;
}

}  // namespace
}  // namespace dress

namespace dress {
namespace {

constexpr int NA_MAX_DEVICES = 128;
std::mutex g_na_mu;
unsigned char *g_na_base[NA_MAX_DEVICES];      // device address of the array, per device

// The array's name is a host-side stand-in in host code; its device address
// comes from cudaGetSymbolAddress with the device current.  Outside stream
// capture every call looks it up afresh (a cudaDeviceReset or another
// context made current then cannot leave a stale address behind); while
// `st` is being captured the address of the device's last call outside
// capture is used, so the first call on a device must come before any
// capture.
cudaError_t noalloc_scratch(cudaStream_t st, unsigned char **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= NA_MAX_DEVICES) return cudaErrorInvalidDevice;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) {
        cudaGetLastError();
        cs = cudaStreamCaptureStatusActive;
    }
    std::lock_guard<std::mutex> lk(g_na_mu);
    if (cs == cudaStreamCaptureStatusNone || !g_na_base[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_na_base[dev] = (unsigned char *)p;
    }
    *out = g_na_base[dev];
    return cudaSuccess;
}

}  // namespace
}  // namespace dress

extern "C" int dressx_histogram_noalloc(const double *values, int64_t n, int64_t *pairs, int64_t *num_runs,
                                        void *stream)
{
    using namespace dress;
    if (n < 0 || (n > 0 && (!values || !pairs)) || !num_runs) {
        std::fprintf(stderr, "dress_b200: dressx_histogram_noalloc: bad arguments\n");
        return DRESSX_EINVAL;
    }
    if (n > NOALLOC_MAX) {
        std::fprintf(stderr, "dress_b200: dressx_histogram_noalloc: %lld values exceed the maximum of %lld\n",
                     (long long)n, (long long)NOALLOC_MAX);
        return DRESSX_EUNSUPPORTED;
    }
    cudaStream_t st = (cudaStream_t)stream;
    unsigned char *base = nullptr;
    cudaError_t e = noalloc_scratch(st, &base);
    if (e != cudaSuccess) {
        std::fprintf(stderr, "dress_b200: dressx_histogram_noalloc: scratch address: %s\n", cudaGetErrorString(e));
        return DRESSX_ECUDA;
    }
    if (n == 0) {
        e = cudaMemsetAsync(num_runs, 0, sizeof(int64_t), st);
        return e == cudaSuccess ? DRESSX_OK : DRESSX_ECUDA;
    }
    unsigned long long *A = (unsigned long long *)(base + NA_A);
    unsigned long long *B = (unsigned long long *)(base + NA_B);
    long long *offs = (long long *)(base + NA_OFFS);
    int *counts = (int *)(base + NA_COUNTS);
    Tile *tiles = (Tile *)(base + NA_TILESB);
    long long *heads = (long long *)(base + NA_HEADS);
    long long *tbase = (long long *)(base + NA_BASE);
    long long *seg_begin = (long long *)(base + NA_SEG);
    long long *seg_end = seg_begin + 1;
    int *seg_tile0 = (int *)(seg_begin + 2);
    int *moves = seg_tile0 + 2;
    const int nt = (int)((n + TILE - 1) / TILE);

    // every scratch word read below is written first in this call, so the
    // array needs no clearing between calls
    count_launch(), k_na_setup<<<1, 256, 0, st>>>(n, nt, tiles, seg_begin, seg_end, seg_tile0);
    count_launch(), k_na_load<<<(unsigned)((n + 255) / 256 < 1024 ? (n + 255) / 256 : 1024), 256, 0, st>>>(n, values, A);
    unsigned long long *a = A, *b = B;
    for (int pass = 0; pass < 8; ++pass) {           // even pass count: sorted keys end in A
        const int shift = 8 * pass;
        count_launch(), k_tile_hist<<<nt, HT, 0, st>>>(tiles, a, shift, counts);
        count_launch(), k_seg_offsets<<<1, RADIX, 0, st>>>(seg_begin, seg_tile0, counts, offs, moves);
        count_launch(), k_tile_scatter<<<nt, HT, 0, st>>>(tiles, a, b, shift, offs, nullptr, nullptr);
        unsigned long long *t = a;
        a = b;
        b = t;
    }
    count_launch(), k_tile_heads<<<nt, HT, 0, st>>>(tiles, seg_begin, A, heads);
    count_launch(), k_na_scan<<<1, 32, 0, st>>>(heads, nt, tbase);
    long long *starts = (long long *)B;               // B is free once the keys are sorted into A
    long long *out_pairs = (long long *)pairs;
    count_launch(), k_na_runs<<<nt, HT, 0, st>>>(tiles, A, tbase, starts, out_pairs);
    count_launch(), k_na_counts<<<(unsigned)((n + 255) / 256 < 1024 ? (n + 255) / 256 : 1024), 256, 0, st>>>(
        n, nt, tbase, starts, out_pairs, (long long *)num_runs);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        std::fprintf(stderr, "dress_b200: dressx_histogram_noalloc: launch: %s\n", cudaGetErrorString(e));
        return DRESSX_ECUDA;
    }
    return DRESSX_OK;
}
