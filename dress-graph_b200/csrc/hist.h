// hist.h -- exact histograms of device value segments (hist.cu).
#pragma once
#include <vector>

#include "engine.h"

namespace dress {

// Sorts each segment [begin[s], begin[s]+len[s]) of `keys` (raw double bits)
// and returns, per segment, the flat [value_bits, count, ...] list ascending
// by value with ==-equal values merged.  `alt` is scratch of the same size as
// `keys`; the sorted keys may end up in either buffer.
Status histogram_segments(unsigned long long *keys, unsigned long long *alt, const std::vector<long long> &begin,
                          const std::vector<long long> &len, std::vector<std::vector<long long>> &out,
                          cudaStream_t st, int sms);

}  // namespace dress
