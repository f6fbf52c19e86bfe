// host_par.h -- a parallel loop over host threads, for the host-side phases
// of batched requests: preparing requests, packing parents, copying results
// out.  The pieces must be independent.
#pragma once

#include <algorithm>
#include <atomic>
#include <thread>
#include <vector>

namespace dress {

// Threads for `units` independent pieces of host work: the machine's hardware
// threads, at most 16, at most one per piece, at least one.
inline int host_threads(long long units)
{
    const unsigned hc = std::thread::hardware_concurrency();
    long long t = hc ? (long long)hc : 4;
    t = std::min<long long>(t, 16);
    t = std::min<long long>(t, units);
    return (int)std::max<long long>(t, 1);
}

// fn(i) for every i in [0, n): `grain` consecutive indices at a time, handed
// out on demand to `threads` threads, the calling thread among them.
template <class F>
void parallel_for(long long n, int threads, F fn, long long grain = 1)
{
    if (n <= 0) return;
    if (grain < 1) grain = 1;
    if (threads <= 1 || n <= grain) {
        for (long long i = 0; i < n; ++i) fn(i);
        return;
    }
    std::atomic<long long> next{0};
    auto work = [&] {
        for (;;) {
            const long long b = next.fetch_add(grain);
            if (b >= n) return;
            const long long e = std::min(n, b + grain);
            for (long long i = b; i < e; ++i) fn(i);
        }
    };
    std::vector<std::thread> th;
    for (int t = 1; t < threads; ++t) th.emplace_back(work);
    work();
    for (auto &t : th) t.join();
}

}  // namespace dress
