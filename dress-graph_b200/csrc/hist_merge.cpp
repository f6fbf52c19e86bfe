// hist_merge.cpp -- merge of exact histograms computed on disjoint shards.
//
// Reference: the MPI layer gathers every rank's flat [value_bits, count]
// histogram and re-inserts the pairs into one hash table
// (libdress/src/mpi/dress_mpi.c:90-118 with dress_hist_add_count,
// libdress/src/dress_histogram.c:62-81), then flattens it ascending by value
// (dress_histogram.c:124-155).  Every shard's list here is already sorted and
// run-length encoded, so one k-way merge over the order-preserving integer
// image of the values gives the same list: counts of equal bit patterns are
// added (the map's key; a NaN never equals an entry and stays apart), as in
// the device histogram.
#include <cstdlib>
#include <cstring>
#include <queue>
#include <vector>

#include "engine.h"

namespace dress {
namespace {

inline unsigned long long ordered(long long bits)
{
    unsigned long long b = (unsigned long long)bits;
    return (b >> 63) ? ~b : (b | 0x8000000000000000ULL);
}

inline double as_double(long long bits)
{
    double d;
    std::memcpy(&d, &bits, sizeof d);
    return d;
}

}  // namespace
}  // namespace dress

using namespace dress;

extern "C" int dressx_hist_merge(const int64_t *const *flats, const int64_t *lens, int n, int64_t **out,
                                 int64_t *out_len)
{
    if (!out || !out_len || n < 0 || (n > 0 && (!flats || !lens))) {
        set_last_error(Status::Err(DRESSX_EINVAL, "dressx_hist_merge: bad arguments"));
        return DRESSX_EINVAL;
    }
    *out = nullptr;
    *out_len = 0;
    long long total = 0;
    for (int i = 0; i < n; ++i) {
        if (lens[i] < 0 || (lens[i] & 1) || (lens[i] > 0 && !flats[i])) {
            set_last_error(Status::Err(DRESSX_EINVAL, "dressx_hist_merge: a list is not [bits, count] pairs"));
            return DRESSX_EINVAL;
        }
        total += lens[i];
    }
    if (total == 0) return DRESSX_OK;
    int64_t *res = (int64_t *)std::malloc((size_t)total * sizeof(int64_t));
    if (!res) {
        set_last_error(Status::Err(DRESSX_ENOMEM, "dressx_hist_merge: host allocation failed"));
        return DRESSX_ENOMEM;
    }
    // (ordered key, list) min-heap; ties go to the lower list index
    using Item = std::pair<unsigned long long, int>;
    std::priority_queue<Item, std::vector<Item>, std::greater<Item>> heap;
    std::vector<long long> pos((size_t)n, 0);
    for (int i = 0; i < n; ++i)
        if (lens[i] > 0) heap.push({ordered(flats[i][0]), i});
    long long m = 0;
    while (!heap.empty()) {
        const int i = heap.top().second;
        heap.pop();
        const long long bits = flats[i][pos[(size_t)i]];
        const long long cnt = flats[i][pos[(size_t)i] + 1];
        if (m > 0 && res[m - 2] == bits && as_double(bits) == as_double(bits)) {
            res[m - 1] += cnt;
        } else {
            res[m] = bits;
            res[m + 1] = cnt;
            m += 2;
        }
        pos[(size_t)i] += 2;
        if (pos[(size_t)i] < lens[i]) heap.push({ordered(flats[i][pos[(size_t)i]]), i});
    }
    *out = res;
    *out_len = m;
    return DRESSX_OK;
}
