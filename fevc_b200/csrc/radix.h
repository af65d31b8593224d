// Stable LSD radix sort of (key, payload) pairs, host side.
#pragma once

#include <cstdint>
#include <vector>

namespace fevcb {

// Stable LSD radix sort of (key, payload) pairs by key, 8-bit digits; digits
// in which every key agrees are skipped.  Equal keys keep their input order.
inline void radix_sort_pairs(std::vector<uint64_t>& key, std::vector<uint32_t>& val) {
  size_t n = key.size();
  if (n < 2) return;
  uint64_t all_or = 0, all_and = ~uint64_t(0);
  for (uint64_t k : key) {
    all_or |= k;
    all_and &= k;
  }
  uint64_t varying = all_or ^ all_and;
  std::vector<uint64_t> k2(n);
  std::vector<uint32_t> v2(n);
  for (int shift = 0; shift < 64; shift += 8) {
    if (((varying >> shift) & 0xff) == 0) continue;
    size_t count[257] = {0};
    for (uint64_t k : key) count[((k >> shift) & 0xff) + 1]++;
    for (int b = 0; b < 256; ++b) count[b + 1] += count[b];
    for (size_t i = 0; i < n; ++i) {
      size_t at = count[(key[i] >> shift) & 0xff]++;
      k2[at] = key[i];
      v2[at] = val[i];
    }
    key.swap(k2);
    val.swap(v2);
  }
}

}  // namespace fevcb
