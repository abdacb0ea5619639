// Warp-cooperative building blocks shared by the counting and set-operation
// kernels.  They restate, B200-first, what include/ops/{Search,Intersection}.cuh
// of the reference provide:
//   - shared-memory hash sets probed by every lane (the replacement for
//     per-key global binary searches, Intersection.cuh:56-71);
//   - a flattened ("load-balanced") walk over many short lists so that all 32
//     lanes stay busy when lists are shorter than a warp (the reference idles
//     lanes beyond |sA|, Intersection.cuh:130);
//   - the two-phase cached binary search (Search.cuh:93-138) with a larger,
//     CTA-wide sample cache and 64-bit index arithmetic (the reference's int32
//     `i*size/N` overflows for lists >= 2^26, Intersection.cuh:256,291).
#pragma once
#include <cstdint>

#include "internal.cuh"

namespace gary {

constexpr uint32_t kHashMul = 0x9E3779B1u;  // Fibonacci hashing

__device__ __forceinline__ uint32_t hash_slot(uint32_t x, uint32_t shift) {
  return (x * kHashMul) >> shift;
}

// log2 of the table size for `items` keys: T >= 2*items, T >= 32.
__device__ __forceinline__ int hash_log2(uint32_t items) {
  int l = items > 1 ? 32 - __clz(2 * items - 1) : 1;
  return l < 5 ? 5 : l;
}

// The owners of a flattened walk's positions, batch after batch: segment k
// (lane k's) covers [excl_k, excl_k + len_k) of the concatenation, and the
// walk visits positions pb + lane for pb = 0, 32, 64, ... in order.  Every
// segment sets the bit of its start inside (pb, pb + 32]; one OR across the
// warp gives all of them, and the owner of pb + lane is the owner of pb moved
// on by the starts at or before it.  Precondition: no empty segment before
// the last non-empty one (trailing empty segments start at the total, which
// no position reaches).  All 32 lanes must call owner() for every batch.
struct WarpOwners {
  uint32_t excl, below, base;
  __device__ __forceinline__ WarpOwners(uint32_t excl_, int lane)
      : excl(excl_), below((1u << lane) - 1u), base(0) {}
  __device__ __forceinline__ uint32_t owner(uint32_t pb) {
    const uint32_t d = excl - pb - 1u;
    const uint32_t starts = __reduce_or_sync(kFull, d < 32u ? 1u << d : 0u);
    const uint32_t own = base + __popc(starts & below);
    base += __popc(starts);
    return own;
  }
};

// Index of the k-th set bit (k from 0) of m, for k < popc(m).
__device__ __forceinline__ uint32_t nth_set_bit(uint32_t m, uint32_t k) {
  uint32_t pos = 0;
#pragma unroll
  for (uint32_t w = 16; w; w >>= 1) {
    const uint32_t c = __popc((m >> pos) & ((1u << w) - 1u));
    if (k >= c) {
      k -= c;
      pos += w;
    }
  }
  return pos;
}

// WarpOwners for segments that may be empty anywhere: only non-empty
// segments set start bits, so the count of starts at or before a position is
// its owner's rank among the non-empty segments, and lane r holds the lane of
// the r-th of them.  All 32 lanes must construct and call owner() together.
struct WarpRuns {
  uint32_t excl, below, base, lane_of;
  bool live;
  __device__ __forceinline__ WarpRuns(uint32_t excl_, uint32_t len, int lane)
      : excl(excl_), below((1u << lane) - 1u), base(0), live(len != 0) {
    lane_of = nth_set_bit(__ballot_sync(kFull, live), (uint32_t)lane);
  }
  __device__ __forceinline__ uint32_t owner(uint32_t pb) {
    const uint32_t d = excl - pb - 1u;
    const uint32_t starts = __reduce_or_sync(kFull, live && d < 32u ? 1u << d : 0u);
    const uint32_t rank = base + __popc(starts & below);
    base += __popc(starts);
    return __shfl_sync(kFull, lane_of, rank);
  }
};

__device__ __forceinline__ uint32_t warp_inclusive_sum(uint32_t x, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t t = __shfl_up_sync(kFull, x, o);
    if (lane >= o) x += t;
  }
  return x;
}

__device__ __forceinline__ float warp_sum_f32(float x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(kFull, x, o);
  return x;
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(kFull, x, o);
  return x;
}

// Two-phase search (Search.cuh:120-138 restated): `cache` holds S samples
// cache[i] = list[i*len/S] (i < S) -- or the whole list when len <= S, in
// which case phase 2 never runs.  Returns 1 when x is in list.
__device__ __forceinline__ uint32_t search_2phase(const uint32_t *list, uint32_t len,
                                                  const uint32_t *cache, uint32_t S, uint32_t x) {
  const uint32_t C = len <= S ? len : S;
  // phase 1: last index with cache[i] <= x
  int lo = 0, hi = (int)C - 1, pos = -1;
  while (lo <= hi) {
    int mid = (lo + hi) >> 1;
    uint32_t v = cache[mid];
    if (v == x) return 1;
    if (v < x) {
      pos = mid;
      lo = mid + 1;
    } else {
      hi = mid - 1;
    }
  }
  if (len <= S || pos < 0) return 0;
  // phase 2: list[(pos)*len/S + 1, (pos+1)*len/S) in global memory
  uint64_t b = (uint64_t)pos * len / S + 1;
  uint64_t e = (uint64_t)(pos + 1) * len / S;
  while (b < e) {
    uint64_t mid = (b + e) >> 1;
    uint32_t v = list[mid];
    if (v == x) return 1;
    if (v < x)
      b = mid + 1;
    else
      e = mid;
  }
  return 0;
}

// ---- shared-memory sets over a sorted list -------------------------------
// All three answer contains(x) for x anywhere in [0, 2^32): values outside
// [lo, lo + span] (including the UINT32_MAX padding) are rejected first.

// Bitmap over [lo, lo + span]; branch-free probe.  The word after the
// bitmap is a zero guard: an out-of-range value reads the guard (or the
// never-set tail bits of the last word) and so tests 0.
struct BitmapSet {
  const uint32_t *mem;
  uint32_t lo, guard;
  __device__ __forceinline__ uint32_t contains(uint32_t x) const {
    const uint32_t o = x - lo;
    const uint32_t w = mem[min(o >> 5, guard)];
    return __funnelshift_r(w, 0u, o) & 1u;  // w >> (o & 31)
  }
};

// Bucketised open addressing: 4-slot buckets read with one 16-byte load.
// Slots of a bucket fill in order, so a bucket with a free last slot ends
// the probe sequence.  The builder never fills more than half the slots (it
// drops keys beyond that and reports kLaunchErrTableFull), so at most half
// the buckets are full and every probe ends at a bucket with a free last
// slot: the loop needs no counter (which would cost the hot probe a register).
struct BucketSet {
  const uint4 *tab;
  uint32_t lo, span, bmask;
  int shift;
  __device__ __forceinline__ uint32_t contains(uint32_t x) const {
    if (x - lo > span) return 0;
    uint32_t b = (x * kHashMul) >> shift;
    while (true) {
      const uint4 q = tab[b];
      if (q.x == x || q.y == x || q.z == x || q.w == x) return 1;
      if (q.w == kSentinel) return 0;
      b = (b + 1) & bmask;
    }
  }
};

// Sorted copy (or samples) of the list in shared memory; two-phase search.
struct SearchSet {
  const uint32_t *list, *cache;
  uint32_t len, S, lo, span;
  __device__ __forceinline__ uint32_t contains(uint32_t x) const {
    if (x - lo > span) return 0;
    return search_2phase(list, len, cache, S, x);
  }
};

// Builders: `nthreads` threads (a warp or the CTA) cooperate; `sync`
// separates clear, fill and use.  They need span <= bitmap_max_span(words)
// (bitmap) or d <= words / 2 (buckets) respectively.  A caller that breaks
// the bucket rule gets a table of its first words / 2 keys only and
// kLaunchErrTableFull in *err (when err is not null): a wrong count that is
// reported, never a probe that cannot end.
template <typename Sync>
__device__ __forceinline__ BitmapSet build_bitmap(const uint32_t *__restrict__ av, uint32_t d,
                                                  uint32_t lo, uint32_t span, uint32_t *mem,
                                                  uint32_t tid, uint32_t nthreads, Sync sync) {
  const uint32_t words = (span >> 5) + 2;  // bitmap + zero guard word
  for (uint32_t i = tid; i < words; i += nthreads) mem[i] = 0;
  sync();
  for (uint32_t i = tid; i < d; i += nthreads) {
    const uint32_t o = av[i] - lo;
    if (o <= span) atomicOr(&mem[o >> 5], 1u << (o & 31));  // always true for a sorted list
  }
  sync();
  return BitmapSet{mem, lo, words - 1};
}

// Largest id span a bitmap of `words` shared words covers (guard included).
__host__ __device__ constexpr uint32_t bitmap_max_span(uint32_t words) { return (words - 1) * 32u - 1u; }

template <typename Sync>
__device__ __forceinline__ BucketSet build_buckets(const uint32_t *__restrict__ av, uint32_t d,
                                                   uint32_t lo, uint32_t span, uint32_t *mem,
                                                   uint32_t words, uint32_t tid, uint32_t nthreads,
                                                   Sync sync, unsigned *err) {
  // buckets = next power of two >= d, at most words / 4
  int lb = d > 1 ? 32 - __clz(d - 1) : 0;
  const int cap = 29 - __clz(words);  // log2(words / 4)
  lb = lb < 3 ? 3 : (lb > cap ? cap : lb);
  const uint32_t nb = 1u << lb;
  if (d > 2 * nb) {  // more keys than half the slots
    if (err && tid == 0) atomicOr(err, kLaunchErrTableFull);
    d = 2 * nb;
  }
  for (uint32_t i = tid; i < 4 * nb; i += nthreads) mem[i] = kSentinel;
  sync();
  for (uint32_t i = tid; i < d; i += nthreads) {
    const uint32_t x = av[i];
    uint32_t b = (x * kHashMul) >> (32 - lb);
    bool placed = false;
    for (uint32_t k = 0; k < nb && !placed; ++k) {
      uint32_t *slot = mem + 4 * b;
      placed = atomicCAS(slot, kSentinel, x) == kSentinel || atomicCAS(slot + 1, kSentinel, x) == kSentinel ||
               atomicCAS(slot + 2, kSentinel, x) == kSentinel || atomicCAS(slot + 3, kSentinel, x) == kSentinel;
      b = (b + 1) & (nb - 1);
    }
    if (!placed && err) atomicOr(err, kLaunchErrTableFull);
  }
  sync();
  return BucketSet{reinterpret_cast<const uint4 *>(mem), lo, span, nb - 1, 32 - lb};
}

}  // namespace gary
