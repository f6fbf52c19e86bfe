// hist.h -- exact histograms of device value segments (hist.cu).
#pragma once
#include <vector>

#include "engine.h"

namespace dress {

// Histogram runs left in device memory: pairs[2r], pairs[2r+1] = (value
// bits, count) of run r; run_seg[r] = its segment; runs are grouped by
// segment in segment order.
struct HistResult {
    DevBuf<long long> pairs;
    DevBuf<int> run_seg;
    long long R = 0;
    int nseg = 0;
};

Status histogram_device(unsigned long long *keys, unsigned long long *alt, const std::vector<long long> &begin,
                        const std::vector<long long> &len, HistResult &res, cudaStream_t st, int sms);
Status histogram_download(HistResult &res, std::vector<std::vector<long long>> &out, cudaStream_t st);
// Same results straight into malloc'd per-segment arrays (outs[s], lens[s]
// int64 entries; NULL and 0 for an empty segment; the caller frees them),
// through the pinned staging buffer when one is given.  pre/cap (nullable):
// malloc'd arrays that already exist per segment and their capacity in
// int64 entries; a segment that fits takes its array (trimmed to length,
// the entry cleared), the others get new ones.  Large results are copied
// out by up to max_threads host threads.
Status histogram_fetch(HistResult &res, std::vector<int64_t *> &outs, std::vector<long long> &lens, Pinned *stage,
                       cudaStream_t st, int sms, std::vector<int64_t *> *pre = nullptr,
                       const std::vector<long long> *cap = nullptr, int max_threads = 16);

// Stable ascending sort of n unsigned 64-bit keys with a 32-bit payload
// (LSD radix, 8-bit digits; digits equal on every key are skipped).  The
// results are in whichever buffer of each pair the last pass wrote.  Keys
// known to be below 2^key_bits take only the passes over those bits.
Status sort_pairs(unsigned long long *keys, unsigned long long *alt, unsigned *vals, unsigned *valt, long long n,
                  unsigned long long **sorted_keys, unsigned **sorted_vals, cudaStream_t st, int sms,
                  int key_bits = 64);

// Sorts each segment [begin[s], begin[s]+len[s]) of `keys` (raw double bits,
// replaced by their order-preserving image, see ordered_to_double) ascending;
// *sorted is whichever of keys / alt holds the result.
Status segmented_sort(unsigned long long *keys, unsigned long long *alt, const std::vector<long long> &begin,
                      const std::vector<long long> &len, unsigned long long **sorted, cudaStream_t st, int sms);

// Sorts each segment [begin[s], begin[s]+len[s]) of `keys` (raw double bits)
// and returns, per segment, the flat [value_bits, count, ...] list ascending
// by value with ==-equal values merged.  `alt` is scratch of the same size as
// `keys`; the sorted keys may end up in either buffer.
Status histogram_segments(unsigned long long *keys, unsigned long long *alt, const std::vector<long long> &begin,
                          const std::vector<long long> &len, std::vector<std::vector<long long>> &out,
                          cudaStream_t st, int sms);

}  // namespace dress
