// Host sorting used by the symbolic setup of triplet patterns (LinearBase::update_sparse).
#pragma once
#include <cstdint>
#include <vector>

namespace vfv {

// Stable LSD radix sort of (key, idx) pairs by the low `bits` bits of key, 16 bits per pass.
// Passes are parallel (OpenMP): each thread histograms and then scatters its own contiguous chunk,
// with the per-(digit, thread) offsets taken in chunk order, so the result is the stable order,
// the same for any thread count.
void radix_sort_pairs(std::vector<uint64_t>& key, std::vector<int64_t>& idx, int bits);

}  // namespace vfv
