// Seeded synthetic generators.  Counter-based (splitmix64 finalizer): sample i
// depends only on (seed, i), so the host and the device produce identical
// edges and any range can be regenerated on the host to check a device batch.
//
// RMAT: (a,b,c,d) = (0.57, 0.19, 0.19, 0.05), no noise, no vertex permutation;
// each level picks a quadrant by comparing a 32-bit draw with integer
// thresholds floor(2^32 * {0.57, 0.76, 0.95}), so no floating point is
// involved and both sides agree bit for bit.
// ER: G(n, m) as m distinct unordered non-loop pairs, drawn in order.
#include <cstdint>
#include <unordered_set>
#include <vector>

#include "internal.cuh"

namespace gary {

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

constexpr uint64_t kGolden = 0x9E3779B97F4A7C15ull;
constexpr uint32_t kRmatA = (uint32_t)((57ull << 32) / 100);  // 0.57
constexpr uint32_t kRmatB = (uint32_t)((76ull << 32) / 100);  // 0.57 + 0.19
constexpr uint32_t kRmatC = (uint32_t)((95ull << 32) / 100);  // + 0.19

__host__ __device__ __forceinline__ void rmat_edge(int scale, uint64_t key, uint64_t i,
                                                   uint32_t *s, uint32_t *d) {
  uint32_t src = 0, dst = 0;
  for (int l = 0; l < scale; l += 2) {
    const uint64_t r = mix64(key + (i * 16 + (uint64_t)(l >> 1)) * kGolden);
    for (int h = 0; h < 2 && l + h < scale; ++h) {
      const uint32_t x = h ? (uint32_t)(r >> 32) : (uint32_t)r;
      const uint32_t sb = x >= kRmatB;
      const uint32_t db = (x >= kRmatA && x < kRmatB) || x >= kRmatC;
      src = (src << 1) | sb;
      dst = (dst << 1) | db;
    }
  }
  *s = src;
  *d = dst;
}

inline uint64_t rmat_key(uint64_t seed) { return mix64(seed ^ 0x5851F42D4C957F2Dull); }

__global__ void k_rmat(int scale, uint64_t key, uint64_t first, uint64_t count,
                       uint32_t *__restrict__ src, uint32_t *__restrict__ dst) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count;
       i += (uint64_t)gridDim.x * blockDim.x)
    rmat_edge(scale, key, first + i, &src[i], &dst[i]);
}

}  // namespace gary

extern "C" int gary_gen_rmat(int scale, uint64_t seed, uint64_t first, uint64_t count,
                             uint32_t *src, uint32_t *dst) {
  GARY_CHECK_ARG(scale >= 1 && scale <= 31, "scale must be in [1, 31]");
  GARY_CHECK_ARG(count == 0 || (src && dst), "src/dst is NULL");
  const uint64_t key = gary::rmat_key(seed);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)count; ++i)
    gary::rmat_edge(scale, key, first + (uint64_t)i, &src[i], &dst[i]);
  return GARY_OK;
}

extern "C" int gary_gen_rmat_device(int scale, uint64_t seed, uint64_t first, uint64_t count,
                                    uint32_t *d_src, uint32_t *d_dst, void *stream) {
  GARY_CHECK_ARG(scale >= 1 && scale <= 31, "scale must be in [1, 31]");
  GARY_CHECK_ARG(count == 0 || (d_src && d_dst), "src/dst is NULL");
  if (!count) return GARY_OK;
  uint64_t blocks = (count + 255) / 256;
  uint64_t cap = (uint64_t)gary::sm_count() * 32;
  gary::k_rmat<<<(unsigned)(blocks < cap ? blocks : cap), 256, 0, gary::as_stream(stream)>>>(
      scale, gary::rmat_key(seed), first, count, d_src, d_dst);
  GARY_CUDA(cudaGetLastError());
  return GARY_OK;
}

extern "C" int gary_gen_er(uint32_t n, uint64_t m, uint64_t seed, uint32_t *src, uint32_t *dst) {
  GARY_CHECK_ARG(n >= 2, "n must be >= 2");
  GARY_CHECK_ARG(m <= (uint64_t)n * (n - 1) / 2, "m exceeds n(n-1)/2");
  GARY_CHECK_ARG(m == 0 || (src && dst), "src/dst is NULL");
  const uint64_t key = gary::mix64(seed ^ 0x2545F4914F6CDD1Dull);
  std::unordered_set<uint64_t> seen;
  seen.reserve(m * 2);
  uint64_t k = 0, got = 0;
  while (got < m) {
    const uint64_t r = gary::mix64(key + (k++) * gary::kGolden);
    uint32_t a = (uint32_t)(((r & 0xFFFFFFFFull) * n) >> 32);
    uint32_t b = (uint32_t)(((r >> 32) * n) >> 32);
    if (a == b) continue;
    if (a > b) {
      uint32_t t = a;
      a = b;
      b = t;
    }
    if (!seen.insert(((uint64_t)a << 32) | b).second) continue;
    src[got] = a;
    dst[got] = b;
    ++got;
  }
  return GARY_OK;
}

// Barabasi-Albert: a K_{m+1} seed clique, then every new vertex attaches to m
// distinct earlier vertices chosen with probability proportional to degree
// (uniform draws from the list holding each vertex once per incident edge
// end).  Counter-based draws keyed by (seed, draw index).  Writes the edges
// (once each) and their number.
extern "C" int gary_gen_ba(uint32_t n, uint32_t m, uint64_t seed, uint32_t *src, uint32_t *dst,
                           uint64_t *count) {
  GARY_CHECK_ARG(m >= 1 && n > m, "need 1 <= m < n");
  GARY_CHECK_ARG(src && dst && count, "NULL argument");
  const uint64_t key = gary::mix64(seed ^ 0x632BE59BD9B4E019ull);
  std::vector<uint32_t> ends;
  ends.reserve(2ull * ((uint64_t)m * (m + 1) / 2 + (uint64_t)(n - m - 1) * m));
  uint64_t e = 0;
  for (uint32_t a = 0; a <= m; ++a)
    for (uint32_t b = a + 1; b <= m; ++b) {
      src[e] = a;
      dst[e] = b;
      ++e;
      ends.push_back(a);
      ends.push_back(b);
    }
  uint64_t draw = 0;
  std::vector<uint32_t> pick(m);
  for (uint32_t v = m + 1; v < n; ++v) {
    uint32_t got = 0;
    while (got < m) {
      const uint64_t r = gary::mix64(key + (draw++) * gary::kGolden);
      const uint32_t t = ends[(size_t)(((r >> 32) * ends.size()) >> 32)];
      bool dup = false;
      for (uint32_t k = 0; k < got; ++k) dup |= pick[k] == t;
      if (!dup) pick[got++] = t;
    }
    for (uint32_t k = 0; k < m; ++k) {
      src[e] = v;
      dst[e] = pick[k];
      ++e;
      ends.push_back(v);
      ends.push_back(pick[k]);
    }
  }
  *count = e;
  return GARY_OK;
}
