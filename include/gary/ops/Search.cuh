// Membership search in sorted lists: the shim of the reference's
// include/ops/Search.cuh:10-170, with its names and results.
//
//   linear_search(span, key)                   Search.cuh:10-17
//   linear_search(span, key, warp)             Search.cuh:19-31 (warp-cooperative)
//   binary_search(list, key, size)             Search.cuh:33-46
//   binary_search(indexable, key)              Search.cuh:48-61
//   binary_search(indexable, key, pos)         Search.cuh:63-81: pos = index of
//                                              key, else of the last element
//                                              < key (-1 when none)
//   build_cache(list, cache[, group])          Search.cuh:93-109: cache[i] =
//                                              list[i * size / N]
//   fill_cache(cache, val, group)              Search.cuh:111-116
//   binary_search_2phase(list, cache, key)     Search.cuh:118-138
//   binary_search_2phase(list, cache, key, n)  Search.cuh:140-170: the warp's
//                                              32 cache words sit at
//                                              cache[warp_in_block * 32]
//
// Searches here are lower-bound loops of fixed trip count (ceil log2 n steps,
// no early exit), which keeps a warp's lanes in step.  Bucket bounds are
// computed in 64 bits: the reference's `pos * size / N` in int overflows for
// lists of 2^26 entries and more (Intersection.cuh:256,291).
#pragma once
#include <cooperative_groups.h>

#include "gary/ops/DeviceIterator.cuh"

// first index in [0, n) whose element is >= key (n when none)
template <typename Indexable, typename T>
CUDA_INLINE HOST_DEVICE size_t gary_lower_bound(const Indexable &list, size_t n, T key) {
  size_t base = 0;
  while (n > 1) {
    const size_t half = n >> 1;
    base = (list[base + half - 1] < key) ? base + half : base;
    n -= half;
  }
  return base + (n == 1 && list[base] < key);
}

template <typename T>
CUDA_INLINE HOST_DEVICE int linear_search(Span<T, void> span, std::remove_cv_t<T> key) {
  for (auto v : span)
    if (v >= key) return v == key;
  return 0;
}

// warp-cooperative: the warp reads 32 consecutive elements per step
template <typename T, typename Group>
CUDA_INLINE DEVICE_ONLY int linear_search(Span<T, void> span, std::remove_cv_t<T> key,
                                          const Group &warp) {
  for (size_t base = 0; base < span.size(); base += warp.num_threads()) {
    const size_t i = base + warp.thread_rank();
    const bool in = i < span.size();
    const auto v = in ? span[i] : key;
    if (warp.any(in && v == key)) return 1;
    if (warp.any(in && v > key)) return 0;
  }
  return 0;
}

template <typename T, typename S = std::remove_cv_t<T>>
CUDA_INLINE HOST_DEVICE bool binary_search(T *list, S key, S size) {
  if (size <= 0) return false;
  const size_t i = gary_lower_bound(list, (size_t)size, key);
  return i < (size_t)size && list[i] == key;
}

template <class Indexable, typename T = typename Indexable::value_type>
inline HOST_DEVICE bool binary_search(Indexable span, T key) {
  const size_t n = span.size();
  const size_t i = gary_lower_bound(span, n, key);
  return i < n && span[i] == key;
}

template <class Indexable, typename T = typename Indexable::value_type>
inline HOST_DEVICE bool binary_search(Indexable span, T key, int &pos) {
  const size_t n = span.size();
  const size_t i = gary_lower_bound(span, n, key);
  if (i < n && span[i] == key) {
    pos = (int)i;
    return true;
  }
  pos = (int)i - 1;
  return false;
}

template <typename T, size_t N, typename S = std::remove_cv_t<T>>
inline HOST_DEVICE void build_cache(Span<T, void> list, Array<S, N> &cache) {
  const uint64_t size = list.size();
  if (size == 0) return;  // nothing to cache; binary_search_2phase answers false
  for (size_t i = 0; i < N; ++i) cache[i] = list[(size_t)(i * size / N)];
}

template <typename T, size_t N, typename CudaGroup, typename S = std::remove_cv_t<T>>
inline DEVICE_ONLY void build_cache(Span<T, void> list, Array<S, N> &cache, const CudaGroup &g) {
  const uint64_t size = list.size();
  if (size == 0) return;
  for (size_t i = g.thread_rank(); i < N; i += g.num_threads())
    cache[i] = list[(size_t)(i * size / N)];
}

template <typename T, size_t N, typename CudaGroup, typename S = std::remove_cv_t<T>>
inline DEVICE_ONLY void fill_cache(Array<S, N> &cache, T val, const CudaGroup &g) {
  for (size_t i = g.thread_rank(); i < N; i += g.num_threads()) cache[i] = val;
}

// cache = build_cache(list): find the cache bucket of key, then search that
// bucket's slice [pos * size / N, (pos + 1) * size / N) of the list
template <typename T, size_t N, typename S = std::remove_cv_t<T>>
inline HOST_DEVICE bool binary_search_2phase(Span<T, void> list, const Array<S, N> &cache, S key) {
  const uint64_t size = list.size();
  if (size == 0) return false;
  int pos = 0;
  if (binary_search(cache, key, pos)) return true;
  if (pos < 0) return false;
  const uint64_t lo = (uint64_t)pos * size / N, hi = (uint64_t)(pos + 1) * size / N;
  const size_t i = gary_lower_bound(list.begin() + lo, (size_t)(hi - lo), key);
  return lo + i < hi && list[lo + i] == key;
}

// warp-level form: 32 cache words per warp of the block, at cache[w * 32]
template <typename T>
CUDA_INLINE DEVICE_ONLY bool binary_search_2phase(T *list, T *cache, T key, T size) {
  namespace cg = cooperative_groups;
  const unsigned w = (unsigned)(cg::this_thread_block().thread_rank() / WARP_SIZE);
  const Array<T, WARP_SIZE> c(cache + (size_t)w * WARP_SIZE);
  return binary_search_2phase(Span<T, void>(list, (size_t)size), c, key);
}
