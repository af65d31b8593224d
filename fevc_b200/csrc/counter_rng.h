// VCKSS-COUNTER-V1: Philox4x64-10 keyed by SplitMix64(seed).
//
// Contract (reference rust/RNG_CONTRACT.md:5-41, vckss-core/src/rng.rs:73-93):
//   key     = (splitmix64(seed), splitmix64(seed ^ 0xd1b54a32d192ed03))
//   counter = (entity, probe / 4, word, domain tag); lane = probe % 4
//   10 rounds; the Weyl key bump happens between rounds, not after the last.
//   atom(n) = 2 * popcount(selected bits of ceil(n/64) words) - n.
// The same code compiles for the host and for sm_100a; on the device the
// 64x64->128 products lower to mul.lo/mul.hi.u64.
#pragma once
#include <cstdint>

#if defined(__CUDACC__)
#define FEVCB_HD __host__ __device__ __forceinline__
#else
#define FEVCB_HD inline
#endif

namespace fevcb {

constexpr uint64_t TAG_LEVERAGE = 0x4c45564552414745ull;
constexpr uint64_t TAG_TARGET = 0x0054415247455401ull;
constexpr uint64_t TAG_COMPONENT_INFERENCE = 0x434f4d50494e4601ull;
constexpr uint64_t TAG_COMPONENT_CRITICAL = 0x434f4d5051435201ull;
constexpr uint64_t TAG_COMPONENT_CONTROL = 0x434f4d5043544c01ull;
constexpr uint64_t TAG_COMPONENT_FOLD = 0x434f4d5056464c01ull;
constexpr uint64_t TAG_OBSERVATION_RESIDUAL = 0x4f4253524d4f4d01ull;
constexpr uint64_t TAG_DIAGNOSTIC = 0x444941474e4f5354ull;
constexpr uint64_t TAG_RETRY = 0x0052455452590001ull;
constexpr uint64_t TAG_SELF_TEST = 0x53454c4654455354ull;
constexpr uint64_t MAX_WORDS_PER_ATOM = uint64_t(1) << 20;

FEVCB_HD uint64_t splitmix64(uint64_t x) {
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}

FEVCB_HD void mulhilo64(uint64_t a, uint64_t b, uint64_t& hi, uint64_t& lo) {
#if defined(__CUDA_ARCH__)
  lo = a * b;
  hi = __umul64hi(a, b);
#else
  unsigned __int128 p = (unsigned __int128)a * b;
  lo = (uint64_t)p;
  hi = (uint64_t)(p >> 64);
#endif
}

struct PhiloxKey {
  uint64_t k0, k1;
};

FEVCB_HD PhiloxKey philox_key(uint64_t seed) {
  return PhiloxKey{splitmix64(seed), splitmix64(seed ^ 0xd1b54a32d192ed03ull)};
}

// One Philox4x64-10 block; counter c = (entity, probe_block, word, tag).
FEVCB_HD void philox_block(PhiloxKey key, uint64_t c0, uint64_t c1, uint64_t c2, uint64_t c3,
                           uint64_t out[4]) {
  uint64_t k0 = key.k0, k1 = key.k1;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    uint64_t h0, l0, h1, l1;
    mulhilo64(0xd2b74407b1ce6e93ull, c0, h0, l0);
    mulhilo64(0xca5a826395121157ull, c2, h1, l1);
    uint64_t n0 = h1 ^ c1 ^ k0;
    uint64_t n2 = h0 ^ c3 ^ k1;
    c0 = n0;
    c1 = l1;
    c2 = n2;
    c3 = l0;
    if (r != 9) {
      k0 += 0x9e3779b97f4a7c15ull;
      k1 += 0xbb67ae8584caa73bull;
    }
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

FEVCB_HD int popcount64(uint64_t v) {
#if defined(__CUDA_ARCH__)
  return __popcll(v);
#else
  return __builtin_popcountll(v);
#endif
}

// Rademacher sums for the four lanes of one probe block:
// out[lane] = 2 * popcount - trials for probe = 4 * probe_block + lane.
FEVCB_HD void rademacher_block_sums(PhiloxKey key, uint64_t tag, uint64_t probe_block,
                                    uint64_t entity, uint64_t trials, int64_t out[4]) {
  uint64_t full = trials >> 6, rem = trials & 63;
  int64_t pos[4] = {0, 0, 0, 0};
  uint64_t b[4];
  for (uint64_t w = 0; w < full; ++w) {
    philox_block(key, entity, probe_block, w, tag, b);
#pragma unroll
    for (int l = 0; l < 4; ++l) pos[l] += popcount64(b[l]);
  }
  if (rem) {
    uint64_t mask = (uint64_t(1) << rem) - 1;
    philox_block(key, entity, probe_block, full, tag, b);
#pragma unroll
    for (int l = 0; l < 4; ++l) pos[l] += popcount64(b[l] & mask);
  }
#pragma unroll
  for (int l = 0; l < 4; ++l) out[l] = 2 * pos[l] - (int64_t)trials;
}

// Rademacher sums over the copy range [offset, offset + trials) of one entity:
// copy c draws bit c % 64 of word c / 64 (+1 for a set bit, -1 otherwise),
// for the four probes 4 * probe_block + lane.  offset = 0 reproduces
// rademacher_block_sums.
FEVCB_HD void rademacher_range_block_sums(PhiloxKey key, uint64_t tag, uint64_t probe_block, uint64_t entity,
                                          uint64_t offset, uint64_t trials, int64_t out[4]) {
  int64_t pos[4] = {0, 0, 0, 0};
  uint64_t b[4];
  uint64_t c = offset, end = offset + trials;
  while (c < end) {
    uint64_t word = c >> 6, lo = c & 63, hi = end - (word << 6);
    if (hi > 64) hi = 64;
    uint64_t mask = (hi == 64 ? ~uint64_t(0) : ((uint64_t(1) << hi) - 1)) & ~((uint64_t(1) << lo) - 1);
    philox_block(key, entity, probe_block, word, tag, b);
#pragma unroll
    for (int l = 0; l < 4; ++l) pos[l] += popcount64(b[l] & mask);
    c = (word << 6) + hi;
  }
#pragma unroll
  for (int l = 0; l < 4; ++l) out[l] = 2 * pos[l] - (int64_t)trials;
}

}  // namespace fevcb
