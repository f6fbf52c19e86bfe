// scan.cu -- device-wide exclusive prefix sum (int32/int64 -> int64).
//
// Three launches: per-tile sums, one-block scan of the tile sums, per-tile
// rescan with the tile's offset.  Used by set-up steps (CSR offsets,
// intercept offsets, bin cursors), never inside a sweep.
#include "engine.h"

namespace dress {

namespace {
constexpr int SB = 512;          // threads per scan block
constexpr int SI = 8;            // items per thread
constexpr long long TILE = (long long)SB * SI;

__device__ __forceinline__ long long block_exclusive(long long v, long long *total)
{
    __shared__ long long ws[SB / 32];
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    long long x = v;
    for (int o = 1; o < 32; o <<= 1) {
        long long y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) ws[wid] = x;
    __syncthreads();
    if (wid == 0) {
        long long s = lane < SB / 32 ? ws[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            long long y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < SB / 32) ws[lane] = s;
    }
    __syncthreads();
    long long before = wid > 0 ? ws[wid - 1] : 0;
    *total = ws[SB / 32 - 1];
    __syncthreads();
    return before + x - v;
}

template <class T>
__global__ void k_tile_sums(const T *in, long long n, long long *sums)
{
    long long base = blockIdx.x * TILE + (long long)threadIdx.x * SI;
    long long s = 0;
#pragma unroll
    for (int i = 0; i < SI; ++i)
        if (base + i < n) s += (long long)in[base + i];
    long long tot;
    block_exclusive(s, &tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

__global__ void k_scan_sums(long long *sums, long long nt)
{
    long long carry = 0;
    for (long long c = 0; c < nt; c += TILE) {
        long long base = c + (long long)threadIdx.x * SI;
        long long v[SI];
        long long s = 0;
#pragma unroll
        for (int i = 0; i < SI; ++i) {
            v[i] = base + i < nt ? sums[base + i] : 0;
            s += v[i];
        }
        long long tot;
        long long run = carry + block_exclusive(s, &tot);
#pragma unroll
        for (int i = 0; i < SI; ++i) {
            if (base + i < nt) sums[base + i] = run;
            run += v[i];
        }
        carry += tot;
    }
}

template <class T>
__global__ void k_tile_scan(const T *in, long long *out, long long n, const long long *sums)
{
    long long base = blockIdx.x * TILE + (long long)threadIdx.x * SI;
    long long v[SI];
    long long s = 0;
#pragma unroll
    for (int i = 0; i < SI; ++i) {
        v[i] = base + i < n ? (long long)in[base + i] : 0;
        s += v[i];
    }
    long long tot;
    long long run = sums[blockIdx.x] + block_exclusive(s, &tot);
#pragma unroll
    for (int i = 0; i < SI; ++i) {
        if (base + i < n) out[base + i] = run;
        run += v[i];
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == SB - 1) out[n] = run;
}

template <class T>
Status scan_impl(const T *in, long long *out, long long n, long long *tmp, cudaStream_t st)
{
    if (n <= 0) {
        DRESS_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(long long), st));
        return Status::Ok();
    }
    long long nt = (n + TILE - 1) / TILE;
    count_launch(), k_tile_sums<T><<<(unsigned)nt, SB, 0, st>>>(in, n, tmp);
    count_launch(), k_scan_sums<<<1, SB, 0, st>>>(tmp, nt);
    count_launch(), k_tile_scan<T><<<(unsigned)nt, SB, 0, st>>>(in, out, n, tmp);
    DRESS_CUDA_TRY(cudaGetLastError());
    return Status::Ok();
}
}  // namespace

size_t scan_tmp_elems(long long n) { return (size_t)((n + TILE - 1) / TILE) + 1; }

Status exclusive_scan_i32(const int *in, long long *out, long long n, long long *tmp, cudaStream_t st)
{
    return scan_impl<int>(in, out, n, tmp, st);
}

Status exclusive_scan_i64(const long long *in, long long *out, long long n, long long *tmp, cudaStream_t st)
{
    return scan_impl<long long>(in, out, n, tmp, st);
}

}  // namespace dress
