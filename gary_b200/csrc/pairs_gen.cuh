// Seeded set-intersection pairs (the microbench workload), identical on the
// host and the device: every value is integer arithmetic on a counter hash.
//
// Pair i has lists A and B.  Lengths are Zipf(s) on [1, nmax] drawn by
// inverse CDF from a uint64 threshold table (built once on the host by
// gary_zipf_table, so both sides read the same table).  A list of length L
// holds one value per bucket [b(j), b(j+1)), b(j) = floor(j * R / L), so it
// is sorted and unique in [0, R).  A fraction `overlap` (as a 32-bit
// threshold) of the shorter list's buckets is planted with the longer list's
// value from its first bucket inside that bucket, when one fits.
#pragma once
#include <cstdint>

namespace gary {

__host__ __device__ __forceinline__ uint64_t pmix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

struct PairGen {
  uint64_t key;              // derived from the seed
  uint64_t range;            // R: values in [0, R)
  uint32_t overlap_thresh;   // plant when hash32 < overlap_thresh
  uint32_t nmax;             // Zipf support [1, nmax]
  const uint64_t *cdf;       // nmax thresholds: length k+1 when r < cdf[k]

  __host__ __device__ __forceinline__ uint64_t h(uint64_t a, uint64_t b) const {
    return pmix64(key + pmix64(a * 0x9E3779B97F4A7C15ull + b));
  }
  __host__ __device__ __forceinline__ uint32_t length(uint64_t pair, int side) const {
    const uint64_t r = h(pair, 0xA000000000000000ull + side);
    uint32_t lo = 0, hi = nmax - 1;  // first k with r < cdf[k]
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if (r < cdf[mid]) hi = mid;
      else lo = mid + 1;
    }
    return lo + 1;
  }
  __host__ __device__ __forceinline__ uint64_t bucket(uint64_t j, uint32_t L) const {
    return j * range / L;
  }
  __host__ __device__ __forceinline__ uint32_t base_value(uint64_t pair, int side, uint32_t j,
                                                          uint32_t L) const {
    const uint64_t b0 = bucket(j, L), b1 = bucket(j + 1, L);
    const uint64_t r = h(pair * 2 + side, 0xB000000000000000ull + j);
    return (uint32_t)(b0 + r % (b1 - b0));
  }
  // value j of side `side` of pair `pair`, given both lengths
  __host__ __device__ __forceinline__ uint32_t value(uint64_t pair, int side, uint32_t j,
                                                     uint32_t la, uint32_t lb) const {
    const uint32_t L = side ? lb : la;
    const int short_side = lb < la ? 1 : 0;  // ties: A is the shorter
    if (side == short_side && overlap_thresh) {
      const uint32_t Lg = side ? la : lb;
      const uint32_t hp = (uint32_t)(h(pair, 0xC000000000000000ull + j) >> 32);
      if (hp < overlap_thresh) {
        const uint64_t t = bucket(j, L);
        const uint64_t k = (t * Lg + range - 1) / range;  // first long bucket starting >= t
        if (k < Lg && bucket(k + 1, Lg) <= bucket(j + 1, L))
          return base_value(pair, 1 - side, (uint32_t)k, Lg);
      }
    }
    return base_value(pair, side, j, L);
  }
};

}  // namespace gary
