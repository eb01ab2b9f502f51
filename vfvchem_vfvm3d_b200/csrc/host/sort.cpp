// Parallel stable radix sort of key/index pairs; see sort.hpp.
#include "sort.hpp"

#include <algorithm>
#include <omp.h>

namespace vfv {

void radix_sort_pairs(std::vector<uint64_t>& key, std::vector<int64_t>& idx, int bits) {
    constexpr int kDigits = 1 << 16;
    const int64_t n = (int64_t)key.size();
    if (n < 2) return;
    std::vector<uint64_t> k2(n);
    std::vector<int64_t> i2(n);
    // at least 64 Ki pairs per thread: below that the histograms cost more than the pass
    const int nt = (int)std::max<int64_t>(1, std::min<int64_t>(omp_get_max_threads(), n / 65536));
    std::vector<int64_t> hist((size_t)nt * kDigits);
    for (int shift = 0; shift < bits; shift += 16) {
#pragma omp parallel num_threads(nt)
        {
            const int T = omp_get_num_threads(), t = omp_get_thread_num();
            const int64_t lo = n * t / T, hi = n * (t + 1) / T;
            int64_t* h = &hist[(size_t)t * kDigits];
            std::fill(h, h + kDigits, 0);
            for (int64_t i = lo; i < hi; ++i) h[(key[i] >> shift) & 0xffff]++;
#pragma omp barrier
#pragma omp single
            {
                int64_t run = 0;
                for (int d = 0; d < kDigits; ++d)
                    for (int u = 0; u < T; ++u) {
                        int64_t& c = hist[(size_t)u * kDigits + d];
                        const int64_t v = c;
                        c = run;
                        run += v;
                    }
            }
            for (int64_t i = lo; i < hi; ++i) {
                const int64_t p = h[(key[i] >> shift) & 0xffff]++;
                k2[p] = key[i];
                i2[p] = idx[i];
            }
        }
        key.swap(k2);
        idx.swap(i2);
    }
}

}  // namespace vfv
