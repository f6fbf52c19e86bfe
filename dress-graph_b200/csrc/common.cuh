// common.cuh -- device helpers shared by the B200 DRESS kernels.
//
// Exactness rules (all kernels are compiled with --fmad=false as well):
//   * every product and sum uses the explicit round-to-nearest intrinsics,
//     so no multiply-add is ever fused;
//   * every multi-term sum has the bits of "sort ascending, then sequential
//     Kahan-Babuska-Neumaier" as the reference computes it
//     (libdress/src/dress.c:51-66): either a certified sum in gathering order
//     (CSum below) or, where the certificate fails, that sorted sum itself;
//   * sqrt and division are the IEEE round-to-nearest forms.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define DRESS_INF __longlong_as_double(0x7ff0000000000000ULL)

namespace dress {

__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ double dsqrt(double a) { return __dsqrt_rn(a); }

// One Neumaier step: s <- s + b with the lost low part accumulated in c.
// The larger-magnitude operand is picked by a select rather than a branch:
// the same two operations in the same order as the reference's if/else
// (libdress/src/dress.c:58-62), with no branch in the serial chain.
__device__ __forceinline__ void kbn_step(double &s, double &c, double b)
{
    double t = dadd(s, b);
    bool g = fabs(s) >= fabs(b);
    double big = g ? s : b, small = g ? b : s;
    c = dadd(c, dadd(dsub(big, t), small));
    s = t;
}

// ---- certified sums -----------------------------------------------------------
// The reference sums every item's terms by "sort ascending, then sequential
// Neumaier" (libdress/src/dress.c:51-66).  CSum adds the same terms in ANY
// order (or several partial sums merged in any tree) and then decides, per
// item, whether its result is provably the bits the sorted sum gives:
//
//   s  running sum;  c  sum of the exact rounding errors of every addition
//   into s (Fast2Sum on the larger operand, as the reference's step);
//   a  sum of |x|;  m  smallest term;  n  number of terms.
//
// Whatever the order, s + c equals the exact real sum X of the terms plus
// the rounding error d of the additions into c.  Each error folded into c is
// at most u|t| <= u(1+u)^n a  (u = 2^-53), c takes at most 3n roundings
// (one per term, two per merge), so |d| <= 6.1 n^2 u^2 a for any order -- the
// sorted order included.  Two ways to prove that the sorted sum rounds to
// the same double R = fl(s + c):
//   * exact compensation: all terms positive, every term, partial sum and
//     error a multiple of q = ulp(m), and 2n u a < 2^53 q bounds every
//     partial sum of errors, so every addition into c is exact in any order:
//     d = 0 for both orders, both results are fl(X);
//   * margin: with rho = (s + c) - R computed exactly, the sorted order's
//     pre-rounding value lies within |rho| + 2B of R (B = 16 n^2 u^2 a >= |d|);
//     if that is below the half-gap between R and its nearer neighbour, it
//     rounds to R as well.
// Otherwise (R zero, subnormal or not finite, or a value close to a rounding
// boundary, about 1e-9 of items) result() returns false and the caller sorts.
struct CSum {
    double s, c, a, m;
    int n;
    __device__ __forceinline__ void init()
    {
        s = 0.0;
        c = 0.0;
        a = 0.0;
        m = DRESS_INF;
        n = 0;
    }
    __device__ __forceinline__ void add(double x)
    {
        const double t = dadd(s, x);
        const bool g = fabs(s) >= fabs(x);
        const double big = g ? s : x, small = g ? x : s;
        c = dadd(c, dadd(dsub(big, t), small));
        s = t;
        a = dadd(a, fabs(x));
        m = fmin(m, x);
        ++n;
    }
    __device__ __forceinline__ void merge(double os, double oc, double oa, double om, int on)
    {
        const double t = dadd(s, os);
        const bool g = fabs(s) >= fabs(os);
        const double big = g ? s : os, small = g ? os : s;
        c = dadd(dadd(c, oc), dadd(dsub(big, t), small));
        s = t;
        a = dadd(a, oa);
        m = fmin(m, om);
        n += on;
    }
    // butterfly over the `width` lanes of a group (all lanes end equal)
    __device__ __forceinline__ void merge_lanes(int width)
    {
        for (int o = width >> 1; o > 0; o >>= 1) {
            const double os = __shfl_xor_sync(0xffffffffu, s, o);
            const double oc = __shfl_xor_sync(0xffffffffu, c, o);
            const double oa = __shfl_xor_sync(0xffffffffu, a, o);
            const double om = __shfl_xor_sync(0xffffffffu, m, o);
            const int on = __shfl_xor_sync(0xffffffffu, n, o);
            merge(os, oc, oa, om, on);
        }
    }
    __device__ __forceinline__ bool result(double &out) const
    {
        const double R = dadd(s, c);
        const unsigned long long b = (unsigned long long)__double_as_longlong(R) & 0x7fffffffffffffffULL;
        const int ex = (int)(b >> 52);
        if (ex < 64 || ex > 2000) return false;
        if (m > 0.0) {
            const double mp2 = __longlong_as_double(__double_as_longlong(m) & 0x7ff0000000000000LL);
            if (dmul(dmul((double)n, a), 0x1p-50) < mp2) {
                out = R;
                return true;
            }
        }
        // rho = (s + c) - R exactly (Fast2Sum on the larger operand)
        const bool g = fabs(s) >= fabs(c);
        const double big = g ? s : c, small = g ? c : s;
        const double rho = dadd(dsub(big, R), small);
        double hg = __longlong_as_double((long long)(ex - 53) << 52);
        if ((b & 0xfffffffffffffULL) == 0) hg = dmul(hg, 0.5);
        const double nn = (double)n;
        const double B = dmul(dmul(dmul(nn, nn), 0x1p-102), a);
        if (dadd(fabs(rho), dmul(2.0, B)) < hg) {
            out = R;
            return true;
        }
        return false;
    }
};

// Compare-exchange putting the smaller value at the lower position.
__device__ __forceinline__ void cswap(double &a, double &b)
{
    bool sw = b < a;
    double lo = sw ? b : a;
    double hi = sw ? a : b;
    a = lo;
    b = hi;
}

// Register sorting network on M (power of two) values, ascending.  Bitonic
// network in its single-direction form: for every block size k the first
// comparator pairs i with its mirror i^(k-1), the rest pair i with i^j.
// Missing values are padded with +inf by the caller.
template <int M>
__device__ __forceinline__ void sort_regs(double (&a)[M])
{
#pragma unroll
    for (int k = 2; k <= M; k <<= 1) {
#pragma unroll
        for (int i = 0; i < M; ++i) {
            int j = i ^ (k - 1);
            if (j > i) cswap(a[i], a[j]);
        }
#pragma unroll
        for (int s = k >> 2; s > 0; s >>= 1) {
#pragma unroll
            for (int i = 0; i < M; ++i) {
                int j = i ^ s;
                if (j > i) cswap(a[i], a[j]);
            }
        }
    }
}

// Sorted KBN over the first n (1 <= n <= M) register values.
template <int M>
__device__ __forceinline__ double kbn_regs(const double (&a)[M], int n)
{
    double s = a[0], c = 0.0;
#pragma unroll
    for (int i = 1; i < M; ++i)
        if (i < n) kbn_step(s, c, a[i]);
    return dadd(s, c);
}

// Cooperative in-place ascending sort of buf[0..n) by `nthr` threads with
// index `tid` (a warp or a whole block).  Same single-direction bitonic
// network over the next power of two; comparators whose upper index is
// >= n would compare against a virtual +inf and are skipped.  `sync` is the
// barrier of the cooperating group.
template <class Sync>
__device__ __forceinline__ void sort_shared(double *buf, int n, int tid, int nthr, Sync sync)
{
    int M = 1;
    while (M < n) M <<= 1;
    for (int k = 2; k <= M; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            // each comparator is identified by its lower index i with bit j clear
            int half = M >> 1;
            for (int q = tid; q < half; q += nthr) {
                int i = ((q & ~(j - 1)) << 1) | (q & (j - 1));   // insert a 0 at bit j
                int p = (j == (k >> 1)) ? (i ^ (k - 1)) : (i | j);
                int lo = i < p ? i : p, hi = i < p ? p : i;
                if (hi < n) {
                    double x = buf[lo], y = buf[hi];
                    if (y < x) { buf[lo] = y; buf[hi] = x; }
                }
            }
            sync();
        }
    }
}

// Sequential sorted-KBN over buf[0..n), n >= 1.
__device__ __forceinline__ double kbn_sorted_buf(const double *buf, int n)
{
    double s = buf[0], c = 0.0;
    int i = 1;
    for (; i + 4 <= n; i += 4) {
        double b0 = buf[i], b1 = buf[i + 1], b2 = buf[i + 2], b3 = buf[i + 3];
        kbn_step(s, c, b0);
        kbn_step(s, c, b1);
        kbn_step(s, c, b2);
        kbn_step(s, c, b3);
    }
    for (; i < n; ++i) kbn_step(s, c, buf[i]);
    return dadd(s, c);
}

// Max of a non-negative double over a block, folded into *dst (bits of a
// non-negative double order like unsigned integers).  NaN and 0 are ignored,
// as in the reference's `if (d > max_delta)` update.
__device__ __forceinline__ void block_max_to(unsigned long long *dst, double v)
{
    __shared__ double red[32];
    if (!(v > 0.0)) v = 0.0;
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) red[wid] = v;
    __syncthreads();
    if (wid == 0) {
        int nw = (blockDim.x + 31) >> 5;
        v = lane < nw ? red[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        // most blocks do not raise the running maximum: look before the atomic
        if (lane == 0 && v > 0.0 && v > __longlong_as_double((long long)*(volatile unsigned long long *)dst))
            atomicMax(dst, (unsigned long long)__double_as_longlong(v));
    }
}

__device__ __forceinline__ bool iteration_skipped(const unsigned long long *maxd, int iter, double eps)
{
    return iter > 0 && __longlong_as_double((long long)maxd[iter - 1]) < eps;
}

}  // namespace dress
