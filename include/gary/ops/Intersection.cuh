// Warp-cooperative intersection of sorted lists: the shim of the reference's
// include/ops/Intersection.cuh, same names and return conventions.
//
//   intersectBinarySearch(a, b)              Intersection.cuh:56-71
//   intersectBinarySearch(a, b, cache)       Intersection.cuh:118-135
//   intersectBinarySearch(a, b, out)         Intersection.cuh:18-50
//   intersectBinarySearch(a, b, cache, out)  Intersection.cuh:76-112
//   intersect(a, b[, cache])                 Intersection.cuh:188-199
//   intersect_bs_cache(a, na, b, nb[, c], cache), intersect(a, na, b, nb, cache)
//                                            Intersection.cuh:239-300, 353-359
//
// All 32 lanes of a warp call together (warp-converged).  The shorter list's
// elements are dealt to the lanes in order and each lane searches the longer
// list.  The Span forms return the lane's share of |a & b| (the warp's lanes
// sum to it); the materialising forms write the members to `out` in
// ascending order and still return the lane's share.  Unlike the reference,
// which appends through a shared-memory atomic cursor (unordered, and limited
// to 32 warps a block), the order comes from a ballot prefix: the cursor is a
// warp-uniform register and no shared memory is needed.
#pragma once
#include <cooperative_groups.h>

#include "gary/ops/Search.cuh"

namespace gary_detail {
CUDA_INLINE DEVICE_ONLY unsigned lane_id() { return threadIdx.x & (WARP_SIZE - 1); }

template <typename T>
CUDA_INLINE HOST_DEVICE void order_by_size(Span<T, void> &a, Span<T, void> &b) {
  if (a.size() > b.size()) {
    Span<T, void> t = a;
    a = b;
    b = t;
  }
}

// Deal `a` to the lanes, test each element with `member`, and (when out is not
// null) append the members in order.  Returns the lane's count.
template <typename T, typename Member>
CUDA_INLINE DEVICE_ONLY int probe_all(Span<T, void> a, Member member, std::remove_cv_t<T> *out) {
  const unsigned lane = lane_id();
  int mine = 0;
  size_t cursor = 0;
  for (size_t base = 0; base < a.size(); base += WARP_SIZE) {
    const size_t i = base + lane;
    bool hit = false;
    std::remove_cv_t<T> key{};
    if (i < a.size()) {
      key = a[i];
      hit = member(key);
    }
    mine += hit;
    if (out) {
      const unsigned ballot = __ballot_sync(FULL_MASK, hit);
      if (hit) out[cursor + __popc(ballot & ((1u << lane) - 1))] = key;
      cursor += __popc(ballot);
    }
  }
  __syncwarp();
  return mine;
}
}  // namespace gary_detail

template <typename T = vidT>
inline DEVICE_ONLY int intersectBinarySearch(Span<T, void> sA, Span<T, void> sB) {
  gary_detail::order_by_size(sA, sB);
  return gary_detail::probe_all(sA, [&](std::remove_cv_t<T> k) { return binary_search(sB, k); },
                                (std::remove_cv_t<T> *)nullptr);
}

template <typename T = vidT, size_t N>
inline DEVICE_ONLY int intersectBinarySearch(Span<T, void> sA, Span<T, void> sB,
                                             Array<std::remove_cv_t<T>, N> &cache) {
  gary_detail::order_by_size(sA, sB);
  auto warp = cooperative_groups::tiled_partition<WARP_SIZE>(cooperative_groups::this_thread_block());
  build_cache(sB, cache, warp);
  __syncwarp();
  return gary_detail::probe_all(
      sA, [&](std::remove_cv_t<T> k) { return binary_search_2phase(sB, cache, k); },
      (std::remove_cv_t<T> *)nullptr);
}

template <typename T = vidT, bool OutSorted = true>
inline DEVICE_ONLY int intersectBinarySearch(Span<T, void> sA, Span<T, void> sB,
                                             std::remove_cv_t<T> *out) {
  gary_detail::order_by_size(sA, sB);
  return gary_detail::probe_all(sA, [&](std::remove_cv_t<T> k) { return binary_search(sB, k); }, out);
}

template <typename T = vidT, size_t N, bool OutSorted = true>
inline DEVICE_ONLY int intersectBinarySearch(Span<T, void> sA, Span<T, void> sB,
                                             Array<std::remove_cv_t<T>, N> &cache,
                                             std::remove_cv_t<T> *out) {
  gary_detail::order_by_size(sA, sB);
  auto warp = cooperative_groups::tiled_partition<WARP_SIZE>(cooperative_groups::this_thread_block());
  build_cache(sB, cache, warp);
  __syncwarp();
  return gary_detail::probe_all(
      sA, [&](std::remove_cv_t<T> k) { return binary_search_2phase(sB, cache, k); }, out);
}

template <typename T = vidT, size_t N>
inline DEVICE_ONLY int intersect(Span<T, void> sA, Span<T, void> sB,
                                 Array<std::remove_cv_t<T>, N> &cache) {
  if (sA.size() == 0 || sB.size() == 0) return 0;
  return intersectBinarySearch(sA, sB, cache);
}

template <typename T = vidT>
inline DEVICE_ONLY int intersect(Span<T, void> sA, Span<T, void> sB) {
  if (sA.size() == 0 || sB.size() == 0) return 0;
  return intersectBinarySearch(sA, sB);
}

// Pointer forms.  `cache` holds 32 words per warp of the block
// (cache[warp_in_block * 32 ...]).  With `c`: members written to c in
// ascending order and the warp's total returned to every lane; without: the
// lane's share.
template <typename T = vidT>
CUDA_INLINE DEVICE_ONLY T intersect_bs_cache(T *a, T size_a, T *b, T size_b, T *c, T *cache) {
  if (size_a == 0 || size_b == 0) return 0;
  Span<T, void> sA(a, (size_t)size_a), sB(b, (size_t)size_b);
  Array<T, WARP_SIZE> warp_cache(cache + (threadIdx.x / WARP_SIZE) * WARP_SIZE);
  const int mine = intersectBinarySearch(sA, sB, warp_cache, c);
  int total = mine;
  for (int o = 16; o; o >>= 1) total += __shfl_xor_sync(FULL_MASK, total, o);
  return (T)total;
}

template <typename T = vidT>
CUDA_INLINE DEVICE_ONLY T intersect_bs_cache(T *a, T size_a, T *b, T size_b, T *cache) {
  if (size_a == 0 || size_b == 0) return 0;
  Span<T, void> sA(a, (size_t)size_a), sB(b, (size_t)size_b);
  Array<T, WARP_SIZE> warp_cache(cache + (threadIdx.x / WARP_SIZE) * WARP_SIZE);
  return (T)intersectBinarySearch(sA, sB, warp_cache);
}

// As in the reference (Intersection.cuh:354-359), the fifth argument is the
// warp caches (32 words per warp), and the result is the lane's share.
template <typename T = vidT>
CUDA_INLINE DEVICE_ONLY T intersect(T *a, T size_a, T *b, T size_b, T *c) {
  return intersect_bs_cache(a, size_a, b, size_b, c);
}

// ---- bounded / ancestor-filtered counts -----------------------------------
// The intersect_num family the reference leaves commented out
// (Intersection.cuh:361-485), for pattern matching with symmetry breaking:
// the lane's share of |{x in a & b : x < upper_bound, x not an ancestor}|.
// Both lists are cut at the bound first (the reference stops its loop at the
// first key past the bound), then the shorter one is searched in the longer.
namespace gary_detail {
template <typename T, typename Keep>
CUDA_INLINE DEVICE_ONLY T count_bounded(T *a, T size_a, T *b, T size_b, T upper_bound, Keep keep) {
  Span<T, void> sa(a, (size_t)size_a), sb(b, (size_t)size_b);
  sa = Span<T, void>(a, gary_lower_bound(sa, sa.size(), upper_bound));
  sb = Span<T, void>(b, gary_lower_bound(sb, sb.size(), upper_bound));
  if (sa.size() == 0 || sb.size() == 0) return 0;
  order_by_size(sa, sb);
  return (T)probe_all(sa, [&](std::remove_cv_t<T> k) { return keep(k) && binary_search(sb, k); },
                      (std::remove_cv_t<T> *)nullptr);
}
}  // namespace gary_detail

template <typename T = vidT>
CUDA_INLINE DEVICE_ONLY T intersect_num(T *a, T size_a, T *b, T size_b) {
  return gary_detail::count_bounded(a, size_a, b, size_b, (T)~(T)0, [](T) { return true; });
}

template <typename T = vidT>
CUDA_INLINE DEVICE_ONLY T intersect_num(T *a, T size_a, T *b, T size_b, T upper_bound) {
  return gary_detail::count_bounded(a, size_a, b, size_b, upper_bound, [](T) { return true; });
}

template <typename T = vidT>
CUDA_INLINE DEVICE_ONLY T intersect_num(T *a, T size_a, T *b, T size_b, T upper_bound, T ancestor) {
  return gary_detail::count_bounded(a, size_a, b, size_b, upper_bound,
                                    [&](T k) { return k != ancestor; });
}

template <typename T = vidT>
CUDA_INLINE DEVICE_ONLY T intersect_num(T *a, T size_a, T *b, T size_b, T *ancestor, int n) {
  return gary_detail::count_bounded(a, size_a, b, size_b, (T)~(T)0, [&](T k) {
    for (int j = 0; j < n; ++j)
      if (k == ancestor[j]) return false;
    return true;
  });
}
