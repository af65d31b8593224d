// Stable LSD radix sort of (key, payload) pairs, host side.
#pragma once

#include <cstdint>
#include <vector>

#include <omp.h>

#include <algorithm>

namespace fevcb {

// Stable LSD radix sort of (key, payload) pairs by key, 8-bit digits; digits
// in which every key agrees are skipped.  Equal keys keep their input order.
// Large inputs run each pass on all host cores: every thread histograms its
// contiguous chunk, bins are laid out bin-major and thread-minor, so a
// thread's chunk lands behind the earlier chunks' entries of the same bin and
// the order stays stable.
inline void radix_sort_pairs(std::vector<uint64_t>& key, std::vector<uint32_t>& val) {
  const size_t n = key.size();
  if (n < 2) return;
  uint64_t all_or = 0, all_and = ~uint64_t(0);
  for (uint64_t k : key) {
    all_or |= k;
    all_and &= k;
  }
  const uint64_t varying = all_or ^ all_and;
  std::vector<uint64_t> k2(n);
  std::vector<uint32_t> v2(n);
  const int threads = n >= (size_t(1) << 18) ? std::max(1, omp_get_max_threads()) : 1;
  std::vector<size_t> count(size_t(threads) * 256);
  for (int shift = 0; shift < 64; shift += 8) {
    if (((varying >> shift) & 0xff) == 0) continue;
    std::fill(count.begin(), count.end(), 0);
#pragma omp parallel num_threads(threads)
    {
      const int t = omp_get_thread_num();
      const size_t b = n * t / threads, e = n * (t + 1) / threads;
      size_t* c = count.data() + size_t(t) * 256;
      for (size_t i = b; i < e; ++i) c[(key[i] >> shift) & 0xff]++;
#pragma omp barrier
#pragma omp single
      {
        size_t at = 0;
        for (int d = 0; d < 256; ++d)
          for (int u = 0; u < threads; ++u) {
            size_t x = count[size_t(u) * 256 + d];
            count[size_t(u) * 256 + d] = at;
            at += x;
          }
      }
      for (size_t i = b; i < e; ++i) {
        size_t at = c[(key[i] >> shift) & 0xff]++;
        k2[at] = key[i];
        v2[at] = val[i];
      }
    }
    key.swap(k2);
    val.swap(v2);
  }
}

}  // namespace fevcb
